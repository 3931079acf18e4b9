"""C ABI checks that need no GPU: the library builds and loads, it exports
every entry point include/hdnnp_gpu.h declares, parser errors come back as
status codes (like the reference's stops, hdnnps.f90:62-65,279-292), and a
valid model on a machine without a GPU fails loudly (no CPU fallback)."""
import ctypes as C
import os

import pytest

from conftest import ABX3_DIR, EXAMPLE_DIR, ROOT


@pytest.fixture(scope="module")
def eng(pkg):
    import __graft_entry__

    __graft_entry__.build()
    from hdnnp_b200 import engine

    return engine


def test_exports_every_declared_symbol(eng):
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            names += eng.exported_symbols(os.path.join(ROOT, "include", h))
    assert "hdnnp_energy_and_forces" in names and "hdnnp_model_load_runner" in names
    L = C.CDLL(eng.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def _load(eng, path):
    h = C.c_void_p()
    code = eng.lib().hdnnp_model_load_runner(os.fsencode(path), 0, C.byref(h))
    return code, eng.lib().hdnnp_last_error().decode(), h


def test_parser_errors_are_status_codes(eng, tmp_path):
    code, msg, _ = _load(eng, str(tmp_path / "nope"))
    assert code == 2 and "input.nn not found" in msg
    src = open(os.path.join(EXAMPLE_DIR, "input.nn")).read()
    d = tmp_path / "order"
    d.mkdir()
    (d / "input.nn").write_text(src.replace("number_of_elements 3\nelements N C H", "elements N C H\nnumber_of_elements 3"))
    code, msg, _ = _load(eng, str(d))
    assert code == 2 and "number_of_elements" in msg
    d2 = tmp_path / "type9"
    d2.mkdir()
    (d2 / "input.nn").write_text(src + "\nsymfunction_short H 9 H 0.1 0.0 12.0\n")
    code, msg, _ = _load(eng, str(d2))
    assert code == 2 and "not supported" in msg
    d3 = tmp_path / "scal"
    d3.mkdir()
    for f in os.listdir(EXAMPLE_DIR):
        (d3 / f).write_bytes(open(os.path.join(EXAMPLE_DIR, f), "rb").read())
    lines = (d3 / "scaling.data").read_text().splitlines()
    (d3 / "scaling.data").write_text("\n".join(lines[:10]) + "\n")
    code, msg, _ = _load(eng, str(d3))
    assert code == 2 and "scaling.data" in msg


def _copy_example(tmp_path, name, edit):
    d = tmp_path / name
    d.mkdir()
    for f in os.listdir(EXAMPLE_DIR):
        (d / f).write_bytes(open(os.path.join(EXAMPLE_DIR, f), "rb").read())
    (d / "input.nn").write_text(edit((d / "input.nn").read_text()))
    return str(d)


def test_cutoff_type_other_than_tanh3_is_refused(eng, tmp_path):
    """The reference always evaluates tanh^3 (symmetryFunctions.f90:310-327),
    RuNNer's cutoff_type 2, whatever input.nn says; another value is refused
    with an I/O status instead of loading a potential that would give wrong
    forces.  Type 2 and a file without the keyword get past the parser (on a
    machine without a GPU they then fail at the device upload, status 5)."""
    import torch

    for bad in ("1", "0", "3"):
        d = _copy_example(tmp_path, "ct" + bad, lambda s, b=bad: s.replace("cutoff_type 2", "cutoff_type " + b))
        code, msg, _ = _load(eng, d)
        assert code == 2 and "cutoff_type " + bad in msg and "tanh^3" in msg, (code, msg)
    d = _copy_example(tmp_path, "ctjunk", lambda s: s.replace("cutoff_type 2", "cutoff_type x"))
    code, msg, _ = _load(eng, d)
    assert code == 2 and "cutoff_type" in msg
    ok_codes = (0,) if torch.cuda.is_available() else (5,)
    for name, edit in (("ct2", lambda s: s), ("ctnone", lambda s: s.replace("cutoff_type 2", ""))):
        code, msg, h = _load(eng, _copy_example(tmp_path, name, edit))
        assert code in ok_codes, (name, code, msg)
        if code == 0:
            eng.lib().hdnnp_model_free(h)


def test_no_cpu_fallback_without_gpu(eng):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    code, msg, _ = _load(eng, ABX3_DIR)  # parses fine, then needs the device
    assert code == 5, (code, msg)
    with pytest.raises(eng.HdnnpError):
        eng.Hdnnp.from_runner(EXAMPLE_DIR)
