"""The C ABI library loads without a GPU, exports every symbol include/su2b.h declares, and
rejects invalid arguments before touching a device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "su2b.h")).read()
    return sorted(set(re.findall(r"^SU2B_API [^(]*?\b(su2b_\w+)\(", text, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_symbols()
    for n in ["su2b_ctx_create", "su2b_upload_gauge", "su2b_gauge_energy", "su2b_gauge_force",
              "su2b_hmc_trajectory", "su2b_metropolis_sweep", "su2b_gradient_flow",
              "su2b_solve", "su2b_fermion_force", "su2b_energy_density"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    from su2_b200 import _abi
    lib = _abi.load()
    for n in declared_symbols():
        assert hasattr(lib, n), n
    assert set(_abi.SIGNATURES) == set(declared_symbols())


def test_invalid_geometry_rejected_without_device():
    from su2_b200 import _abi
    lib = _abi.load()
    ctx = ctypes.c_void_p()
    # odd extent, bad ndims, inactive extent != 1, bad group, bad precision, NULL out
    assert lib.su2b_ctx_create(0, 5, 4, 4, 4, 4, 2.0, 1.0, 0, 0, ctypes.byref(ctx)) == _abi.ERR_INVALID
    assert lib.su2b_ctx_create(0, 4, 4, 4, 4, 5, 2.0, 1.0, 0, 0, ctypes.byref(ctx)) == _abi.ERR_INVALID
    assert lib.su2b_ctx_create(0, 4, 4, 2, 4, 3, 2.0, 1.0, 0, 0, ctypes.byref(ctx)) == _abi.ERR_INVALID
    assert lib.su2b_ctx_create(7, 4, 4, 4, 4, 4, 2.0, 1.0, 0, 0, ctypes.byref(ctx)) == _abi.ERR_INVALID
    assert lib.su2b_ctx_create(0, 4, 4, 4, 4, 4, 2.0, 1.0, 9, 0, ctypes.byref(ctx)) == _abi.ERR_INVALID
    assert lib.su2b_ctx_create(0, 4, 4, 4, 4, 4, 2.0, 1.0, 0, 0, None) == _abi.ERR_INVALID
    assert lib.su2b_ctx_destroy(None) == _abi.ERR_INVALID
    # volumes above 2^29 sites, including extents whose product wraps 64 bits (65536^4 = 2^64)
    for dims in ((1024, 1024, 1024, 2), (65536, 65536, 65536, 65536), (2 ** 30, 2, 2, 2)):
        assert lib.su2b_ctx_create(0, *dims, 4, 2.0, 1.0, 0, 0, ctypes.byref(ctx)) == \
            _abi.ERR_INVALID, dims
    assert lib.su2b_ctx_create(1, 2 ** 30, 1, 1, 4, 2, 2.0, 1.0, 0, 0, ctypes.byref(ctx)) == \
        _abi.ERR_INVALID


def test_null_context_is_an_error():
    from su2_b200 import _abi
    lib = _abi.load()
    d = ctypes.c_double()
    assert lib.su2b_gauge_energy(None, 0, ctypes.byref(d)) == _abi.ERR_INVALID
    assert lib.su2b_hmc_trajectory(None, None, None) == _abi.ERR_INVALID
    assert lib.su2b_last_error(None) == b"null context"


def test_product_does_not_link_the_oracle():
    """The CUDA library is self-contained: its dynamic symbol table neither defines nor
    imports an oracle (orc_*) or reference-harness (ref_*) symbol, and it names neither
    checker library among the libraries it needs."""
    import subprocess

    from su2_b200 import _abi
    syms = subprocess.run(["nm", "-D", _abi.LIB_PATH], capture_output=True, text=True,
                          check=True).stdout.split("\n")
    names = [ln.split()[-1] for ln in syms if ln.strip()]
    assert any(n.startswith("su2b_") for n in names)
    assert not [n for n in names if n.startswith(("orc_", "ref_"))]
    dyn = subprocess.run(["readelf", "-d", _abi.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    needed = [ln for ln in dyn.split("\n") if "(NEEDED)" in ln]
    assert not [ln for ln in needed if "su2oracle" in ln or "su2ref" in ln]


@pytest.mark.parametrize("fn", ["su2b_upload_gauge", "su2b_download_gauge"])
def test_transfer_requires_context(fn):
    from su2_b200 import _abi
    lib = _abi.load()
    assert getattr(lib, fn)(None, None) == _abi.ERR_INVALID


def test_launch_shape_tables_agree_with_the_header():
    """The Python tables of launch shapes have one entry per variant the C ABI accepts, and
    the variant counts equal the header's (and the library's) constants."""
    from su2_b200 import _abi
    text = open(os.path.join(ROOT, "include", "su2b.h")).read()
    nf = int(re.search(r"#define SU2B_FORCE_VARIANTS (\d+)", text).group(1))
    nb = int(re.search(r"#define SU2B_BATCH_VARIANTS (\d+)", text).group(1))
    assert _abi.FORCE_VARIANTS == nf == len(_abi.FORCE_SHAPES)
    assert _abi.BATCH_VARIANTS == nb == len(_abi.BATCH_SHAPES)
    src = open(os.path.join(ROOT, "su2_b200", "csrc", "su2b_internal.h")).read()
    assert int(re.search(r"constexpr int FORCE_VARIANTS = (\d+);", src).group(1)) == nf


def test_noalloc_rejects_bad_sizes_before_touching_a_device():
    """su2b_gauge_energy_noalloc validates its geometry on the host: lattices beyond its
    fixed scratch array, extents whose product would wrap, bad ids and NULL buffers are
    refused before any CUDA call (the pointer below is never dereferenced)."""
    from su2_b200 import _abi
    lib = _abi.load()
    p = ctypes.c_void_p(16)
    f = lib.su2b_gauge_energy_noalloc
    assert f(0, 48, 48, 48, 48, 4, p, p, None) == _abi.ERR_INVALID         # 5.3 M sites
    assert f(0, 65536, 65536, 65536, 65536, 4, p, p, None) == _abi.ERR_INVALID  # 2^64
    assert f(1, 2 ** 30, 1, 1, 4, 2, p, p, None) == _abi.ERR_INVALID
    assert f(0, 8, 8, 8, 8, 4, None, p, None) == _abi.ERR_INVALID
    assert f(0, 8, 8, 8, 8, 4, p, None, None) == _abi.ERR_INVALID
    assert f(2, 8, 8, 8, 8, 4, p, p, None) == _abi.ERR_INVALID
    assert f(0, 8, 8, 8, 8, 5, p, p, None) == _abi.ERR_INVALID
    assert f(0, 8, 8, 2, 8, 3, p, p, None) == _abi.ERR_INVALID             # inactive Lz != 1


def test_every_handle_entry_point_refuses_a_null_handle():
    """Each entry point whose first argument is a context, batch or slab handle returns
    SU2B_ERR_INVALID for a NULL handle (zero or NULL for the other arguments) before it
    touches a device; the last_error accessors name the missing handle."""
    from su2_b200 import _abi
    lib = _abi.load()
    checked = 0
    for name, (res, args) in _abi.SIGNATURES.items():
        if not args or args[0] is not _abi._P:
            continue
        vals = [0 if a in (ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_long)
                else 0.0 if a is ctypes.c_double else None for a in args]
        r = getattr(lib, name)(*vals)
        if name.endswith("last_error"):
            assert r.startswith(b"null"), name
        else:
            assert r == _abi.ERR_INVALID, name
        checked += 1
    assert checked > 60
