"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: runs without a GPU)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"\b(mose_gpu_\w+)\s*\(", text)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from mose_b200 import _lib, build
    build.build()
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_measurement_probe_stays_out_of_the_product(lib):
    """The FP64 issue-ceiling probe is a benchmark tool: it lives in its own
    library, not in the ABI a Fortran solver links."""
    from mose_b200 import _lib
    assert not hasattr(lib, "mose_gpu_fp64_peak")
    assert hasattr(_lib.load_probe(), "mose_probe_fp64_peak")


def test_fortran_module_binds_every_entry_point():
    """mose_b200/fortran/mose_gpu_m.f90 has an ISO_C_BINDING interface, bound
    by name, for every entry point the header declares (no Fortran compiler
    is on these machines, so this is a text check of the module)."""
    f90 = (ROOT / "mose_b200" / "fortran" / "mose_gpu_m.f90").read_text()
    bound = set(re.findall(r'bind\(C, name="(mose_gpu_\w+)"\)', f90))
    public = set(re.findall(r"\b(mose_gpu_\w+)\b", " ".join(l for l in f90.splitlines() if "public ::" in l)))
    assert bound == set(declared_functions())
    assert public >= bound


def test_binding_covers_the_header(lib):
    from mose_b200 import _lib
    assert set(_lib.SIGNATURES) == set(declared_functions())


def test_default_config_matches_reference_defaults(lib):
    from mose_b200 import _lib
    cfg = _lib.Config()
    lib.mose_gpu_default_config(C.byref(cfg))
    # Register_Numerics.f90: time-scheme euler, cfl 0.5, time-accurate false, HLLC
    assert cfg.abi_version == _lib.ABI_VERSION
    assert cfg.n_rk == 1 and cfg.cfl == 0.5 and cfg.time_accurate == 0 and cfg.riemann == 0
    assert cfg.nsc == 1 and cfg.gamma == 1.4


def test_create_rejects_bad_configs_without_touching_the_gpu(lib):
    from mose_b200 import _lib
    cfg = _lib.Config()
    lib.mose_gpu_default_config(C.byref(cfg))
    h = C.c_void_p()
    cfg.nsc = 2          # multi-species is off this path
    assert lib.mose_gpu_create(C.byref(cfg), C.byref(h)) == _lib.ERR_UNSUPPORTED
    cfg.nsc = 1
    cfg.abi_version = 99
    assert lib.mose_gpu_create(C.byref(cfg), C.byref(h)) == _lib.ERR_INVALID
    assert not h.value


def test_library_has_no_cpu_fallback():
    """The package fails loudly when the CUDA library is absent."""
    import importlib
    from mose_b200 import _lib
    saved = _lib.LIB_PATH
    try:
        _lib.LIB_PATH = Path("/nonexistent/libmose_gpu.so")
        _lib._lib = None
        with pytest.raises(RuntimeError, match="no CPU fallback"):
            _lib.load()
    finally:
        _lib.LIB_PATH = saved
        _lib._lib = None
        importlib.reload(_lib)
