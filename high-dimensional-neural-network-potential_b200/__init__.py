"""hdnnp_b200: B200-native HDNNP prediction engine (energy, forces, stress).

The compute path is ``lib/libhdnnp_b200.so`` (CUDA kernels for sm_100a behind a
C ABI, declared in ``include/hdnnp_gpu.h``).  This Python package mirrors the
reference's Fortran interface on top of that ABI:

* ``Hdnnp.from_runner(path)``      -> ``parseRuNNerInput`` (hdnnps.f90:34)
* ``Hdnnp.energy_and_forces(ats)``  -> ``hdnnpEnergyAndForces`` (hdnnps.f90:333)
* ``AtStruct``                      -> ``type atStruct`` (atomicStructure.f90:17)
* ``dEdLat_to_stress``              -> ``dEdLat2Stress`` (atomicStructure.f90:679)

Because the directory name contains hyphens, import it through
``__graft_entry__.load_package()``, which registers it as ``hdnnp_b200``.
"""
from . import workloads  # noqa: F401
