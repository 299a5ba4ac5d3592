"""The C ABI library loads without a GPU, exports every function declared in
include/warpsph_b200.h, validates its arguments before touching the device, and the
ctypes mirror of SphParams matches the C layout."""
import ctypes as C
import re
from pathlib import Path

import pytest

from warpsph_b200 import _capi

HEADER = Path(__file__).resolve().parents[1] / "include" / "warpsph_b200.h"


def declared_in_header():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(sph_[a-z0-9_]+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    names = declared_in_header()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes prototypes cover the header
    assert set(names) <= set(_capi.declared_functions()) | {"sph_version", "sph_last_error_string"}


def test_version_and_kernel_constants():
    lib = _capi.lib()
    assert b"sm_100a" in lib.sph_version()
    c, s = C.c_double(), C.c_double()
    assert lib.sph_kernel_constants(2, 2, C.byref(c), C.byref(s)) == 0
    assert abs(c.value - 9 / 3.141592653589793) < 1e-12 and abs(s.value - 2.171240593) < 1e-9
    assert lib.sph_kernel_constants(9, 2, C.byref(c), C.byref(s)) == _capi_err("BAD_ARG")


def _capi_err(name):
    return {"BAD_ARG": -1, "WORKSPACE": -2, "UNSUPPORTED": -8}[name]


def _params(dim=2):
    p = _capi.SphParams()
    p.dim, p.kernel, p.verlet_scale = dim, 2, 1.4
    for a in range(3):
        p.domain_min[a], p.domain_max[a], p.periodic[a] = -0.5, 0.5, 1
    return p


def test_argument_validation_happens_on_the_host():
    lib = _capi.lib()
    p = _params()
    pp = C.cast(C.pointer(p), C.c_void_p)
    # n == 0 is a no-op even with null pointers
    assert lib.sph_density_gather(pp, 0, 0, None, None, None, None, None, None, None, None) == 0
    # null arrays are rejected before any launch
    assert lib.sph_density_gather(pp, 10, 0, None, None, None, None, None, None, None, None) == -1
    assert b"null pointer" in lib.sph_last_error_string()
    # bad dimension / kernel / support mode
    p.dim = 4
    assert lib.sph_crk_volume(pp, 10, None, None, None, None, None, None, None) == -1
    p.dim, p.kernel = 2, 7
    assert lib.sph_crk_volume(pp, 10, None, None, None, None, None, None, None) == -1
    p.kernel = 2
    assert lib.sph_neighbors_workspace_size(pp, -1, 16, C.byref(C.c_int64())) == -1
    ws = C.c_int64()
    assert lib.sph_neighbors_workspace_size(pp, 1000, 4096, C.byref(ws)) == 0 and ws.value > 4096 * 4
    # a workspace smaller than required is refused
    dummy = 256  # never dereferenced: the size check fails first
    rc = lib.sph_neighbors_build(pp, 1000, dummy, dummy, dummy, 16, 4096, dummy, dummy, dummy, dummy, dummy, dummy, dummy,
                                 dummy, 10, dummy, None, None, dummy, None)
    assert rc == -2


def test_params_layout_matches_c():
    from oracle import oracle
    L = oracle.get("f32").lib
    L.oracle_params_layout.restype = C.c_int64
    assert L.oracle_params_layout(0) == C.sizeof(_capi.SphParams)
    assert L.oracle_params_layout(1) == _capi.SphParams.dim.offset
    assert L.oracle_params_layout(2) == _capi.SphParams.kahan.offset
    assert L.oracle_params_layout(3) == _capi.SphParams.target_neighbors.offset
    assert L.oracle_params_layout(4) == _capi.SphParams.energy_scheme.offset


def test_tensors_must_be_cuda():
    import torch
    from warpsph_b200 import ops
    p = _params()
    x = torch.zeros(4, 2)
    with pytest.raises(RuntimeError, match="CUDA"):
        ops.crk_volume(p, x, torch.ones(4), None)


def test_ctypes_prototypes_match_header_arity():
    """Every ctypes prototype has as many arguments as its C declaration."""
    import re
    from pathlib import Path
    from warpsph_b200 import _capi
    h = (Path(__file__).resolve().parents[1] / "include" / "warpsph_b200.h").read_text()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    for name, args in _capi._PROTOS.items():
        m = re.search(r"\b" + name + r"\s*\(([^;]*?)\)\s*;", h, re.S)
        assert m, name
        params = m.group(1).strip()
        n = 0 if params in ("", "void") else len(params.split(","))
        assert n == len(args), (name, n, len(args))


def test_python_call_sites_pass_every_argument():
    """Every call of a C entry point in the package passes exactly the declared number of
    arguments (``*_lists(...)``, ``*_csr(...)`` and ``*rows`` expand to the three CSR
    pointers).  Runs on the source, so it needs no GPU."""
    import ast
    import pathlib
    root = pathlib.Path(_capi.__file__).resolve().parent
    protos = dict(_capi._PROTOS)
    checked = 0
    for path in sorted(root.glob("*.py")):
        tree = ast.parse(path.read_text())
        for node in ast.walk(tree):
            if not (isinstance(node, ast.Call) and isinstance(node.func, ast.Attribute) and node.func.attr in protos):
                continue
            n, known = 0, True
            for a in node.args:
                if isinstance(a, ast.Starred):
                    v = a.value
                    if isinstance(v, ast.Call) and isinstance(v.func, ast.Name) and v.func.id in ("_lists", "_csr"):
                        n += 3
                    elif isinstance(v, ast.Name) and v.id == "rows":
                        n += 3
                    else:
                        known = False
                else:
                    n += 1
            if known:
                assert n == len(protos[node.func.attr]), f"{path.name}:{node.lineno} {node.func.attr}: {n} != {len(protos[node.func.attr])}"
                checked += 1
    assert checked > 30
