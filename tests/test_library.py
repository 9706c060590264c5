"""CPU-side checks of the product library: it loads, exports every entry point include/gpop.h
declares, and its host logic reports errors as status codes (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "gpop.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gpop_[a-z_0-9]+)\s*\(", src)))


def test_header_and_binding_agree():
    import opengpop_b200 as G
    assert sorted(G.EXPORTS) == _declared()


def test_library_exports_every_declared_symbol():
    import opengpop_b200 as G
    lib = C.CDLL(G.LIB_PATH)
    for name in _declared():
        assert hasattr(lib, name), name


def test_binding_loads():
    import opengpop_b200 as G
    lib = G.load_library()
    assert lib.gpop_status_string(0) == b"ok"
    assert lib.gpop_status_string(5) == b"device wait timed out"


def test_missing_data_is_a_data_error(tmp_path):
    import opengpop_b200 as G
    with pytest.raises(G.GpopError) as e:
        G.Context(data_dir=str(tmp_path))
    assert e.value.status == 3 and "JGM3.gfc" in str(e.value)


def test_corrupt_gravity_file_is_a_data_error(tmp_path):
    import shutil
    import opengpop_b200 as G
    for f in os.listdir(G.DATA_DIR):
        if f != "JGM3.gfc" and not f.endswith(".md"):
            shutil.copy(os.path.join(G.DATA_DIR, f), tmp_path / f)
    (tmp_path / "JGM3.gfc").write_text("modelname JGM3\nmax_degree 70\n")  # no end_of_head
    with pytest.raises(G.GpopError) as e:
        G.Context(data_dir=str(tmp_path))
    assert e.value.status == 3 and "end_of_head" in str(e.value)
    (tmp_path / "JGM3.gfc").write_text(
        "earth_gravity_constant 3.9e14\nradius 6.3e6\nmax_degree 4\nend_of_head ===\n"
        "gfct 0 0 1.0 0.0 0 0\n")  # first data line is not a static 'gfc' row
    with pytest.raises(G.GpopError) as e:
        G.Context(data_dir=str(tmp_path))
    assert e.value.status == 3 and "gfc" in str(e.value)


def test_invalid_config_rejected():
    import opengpop_b200 as G
    with pytest.raises(G.GpopError) as e:
        G.Context(n_corrections=0)
    assert e.value.status == 1


def test_no_gpu_fails_loudly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import opengpop_b200 as G
    with pytest.raises(G.GpopError) as e:
        G.Context()
    assert e.value.status == 2
