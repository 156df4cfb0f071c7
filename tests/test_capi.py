"""The C ABI library loads and exports every entry point include/ declares
(no compute: these run without a GPU)."""

import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "diffsoup_b200.h")
LIB = os.path.join(ROOT, "diffsoup_b200", "libdiffsoup_b200.so")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ds_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build libdiffsoup_b200.so first"
    lib = C.CDLL(LIB)
    syms = declared_symbols()
    assert len(syms) >= 24
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_host_only_entry_points():
    lib = C.CDLL(LIB)
    lib.ds_version.restype = C.c_char_p
    assert b"sm_100a" in lib.ds_version()
    lib.ds_tiles_workspace_size.restype = C.c_size_t
    lib.ds_tiles_workspace_size.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int64]
    a = lib.ds_tiles_workspace_size(8, 15000, 20000, 1 << 20)
    b = lib.ds_tiles_workspace_size(8, 15000, 20000, 2 << 20)
    assert b - a >= 4 << 20  # one int per list entry
    lib.ds_depth_test_workspace.restype = C.c_size_t
    lib.ds_depth_test_workspace.argtypes = [C.c_int] * 3
    assert lib.ds_depth_test_workspace(2, 3, 5) == 2 * 3 * 5 * 8


def test_view_table_and_argument_errors():
    from diffsoup_b200 import _core

    lib = _core.lib
    B = 3
    Hs = (C.c_int * B)(48, 17, 800)
    Ws = (C.c_int * B)(64, 33, 800)
    desc = (_core.ViewDesc * B)()
    npix = C.c_int64(0)
    nt = lib.ds_make_view_table(B, Hs, Ws, desc, C.byref(npix))
    assert nt == 3 * 4 + 2 * 3 + 50 * 50
    assert npix.value == 48 * 64 + 17 * 33 + 800 * 800
    assert desc[1].pix_offset == 48 * 64 and desc[2].tile_base == 12 + 6
    Hs[1] = 0
    rc = lib.ds_make_view_table(B, Hs, Ws, desc, C.byref(npix))
    assert rc == 1 and b"size" in lib.ds_last_error()
    # lattice size mismatch is reported like the reference's runtime_error
    rc = lib.ds_multires_triangle_alpha(0, None, 1, 1, 7, None, None, None)
    assert rc == 1 and lib.ds_last_error() == b"Invalid feature size."
    with pytest.raises(RuntimeError, match="Invalid feature size"):
        _core.check(rc)


def test_train_step_binding_argument_errors():
    """ds_train_step's ctypes signature matches the header: an invalid batch is
    rejected on the host with DS_ERR_ARG before any device work."""
    import ctypes as C
    from diffsoup_b200 import step as S
    from diffsoup_b200 import _core

    cfg = S.StepConfig(0, 10, 30, 8, 0, 2, 16, 1, 1, 0.5)
    null = C.c_void_p(0)
    rc = S._L.ds_train_step(C.byref(cfg), null, 0, 0, *([null] * 17), 0, 0, null, null)
    assert rc == 1 and b"bad sizes" in _core.lib.ds_last_error()
    cfg = S.StepConfig(2, 10, 30, 7, 0, 2, 16, 1, 0, 0.5)
    rc = S._L.ds_train_step(C.byref(cfg), null, 4, 100, *([null] * 17), 0, 0, null, null)
    assert rc == 1 and b"unsupported MLP" in _core.lib.ds_last_error()
    assert S.mlp_param_count(8, 16, 1) == 16 * 11 + 16 + 3 * 16 + 3
    assert S.mlp_param_count(16, 64, 2) == 64 * 19 + 64 + 64 * 64 + 64 + 3 * 64 + 3


def test_step_config_matches_the_header():
    """diffsoup_b200.step.StepConfig lays out ds_step_config field for field
    (names, order and 32-bit types), so a change on one side fails here."""
    from diffsoup_b200 import step as S

    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct \{([^}]*)\}\s*ds_step_config;", src).group(1)
    want = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        ctype, names = decl.split(None, 1)
        want += [(n.strip(), ctype) for n in names.split(",")]
    got = [(n, {C.c_int32: "int32_t", C.c_float: "float"}[t]) for n, t in S.StepConfig._fields_]
    assert got == want
    # construction by name sets every field
    cfg = S.StepConfig(B=2, T=3, V=9, C=8, min_level=0, max_level=2, hidden=16, n_layers=1, stochastic=1,
                       thr_const=0.5, frag_records=2.0, precision=1, block_shape=0, view_enc=0, target_u8=1,
                       shade_mode=0)
    assert (cfg.B, cfg.target_u8, cfg.shade_mode) == (2, 1, 0)


def declared_prototypes():
    """name -> list of parameter declarations of every ds_* prototype."""
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(ds_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", src, flags=re.S):
        params = [p.strip() for p in m.group(2).replace("\n", " ").split(",") if p.strip()]
        protos[m.group(1)] = [] if params == ["void"] else params
    return protos


def test_ctypes_signatures_match_the_header():
    """Every binding in diffsoup_b200/_core.py passes as many arguments as
    the header declares, with 64-bit, floating and pointer slots where the
    header has them (an ABI drift between the two would misread arguments)."""
    from diffsoup_b200 import _core

    protos = declared_prototypes()
    checked = 0
    for name, params in protos.items():
        fn = getattr(_core.lib, name)
        if fn.argtypes is None:
            continue
        assert len(fn.argtypes) == len(params), (name, len(fn.argtypes), len(params))
        for arg, decl in zip(fn.argtypes, params):
            if "*" in decl:
                assert arg in (C.c_void_p, C.c_char_p) or issubclass(arg, C._Pointer), (name, decl, arg)
            elif decl.startswith(("int64_t", "size_t")):
                assert arg in (C.c_int64, C.c_size_t), (name, decl, arg)
            elif decl.startswith("double"):
                assert arg is C.c_double, (name, decl, arg)
            elif decl.startswith("float"):
                assert arg is C.c_float, (name, decl, arg)
            elif decl.startswith(("int ", "int32_t")):
                assert arg is C.c_int, (name, decl, arg)
            elif decl.startswith("ds_stream_t"):
                assert arg is C.c_void_p, (name, decl, arg)
        checked += 1
    assert checked >= 30, checked
