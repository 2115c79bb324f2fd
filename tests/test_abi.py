"""The C-ABI library loads and exports every entry point of the header."""
import ctypes
import pathlib
import re

ROOT = pathlib.Path(__file__).resolve().parent.parent


def header_functions():
    text = (ROOT / "include" / "cadmas_gpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:(?:long|unsigned)\s+)*\w+[\s*]+(\w+)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "defined")))


def test_header_lists_entry_points():
    names = header_functions()
    for n in ("cadmas_create", "cadmas_step", "vf_step_gpu_", "cadmas_m1bcgs_dev"):
        assert n in names


def test_library_exports_all(pkg):
    lib = ctypes.CDLL(str(pkg.build_library()))
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(pkg.EXPORTED) <= set(header_functions())


def test_params_layout_matches_header(pkg):
    """The ctypes mirror and the C struct agree on defaults written by the library."""
    p = pkg.default_params()
    assert p.icgmax == 500 and p.cgpara == 0.95 and p.cgepsr == 1e-12
    assert list(p.idamp) == [-1, -1, -1, -1] and p.damp[1][0] == 0.6
    assert p.diag_relres == 0 and p.precond_ti == 0
    assert p.mixed_eps_inner == 1e-5 and p.wait_limit_s == 2.0  # the last two fields
