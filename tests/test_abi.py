"""The C-ABI library loads without a GPU and exports every entry point that
include/ffx.h declares; the ctypes table matches the header. No device calls."""
import ctypes
import re
from pathlib import Path

import pytest

from fluxfx_b200 import _native as N

ROOT = Path(__file__).resolve().parent.parent


def header_functions():
    text = (ROOT / 'include' / 'ffx.h').read_text()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(ffx_[a-z0-9_]+)\s*\(', text)))


def test_header_declares_the_bound_entry_points():
    assert header_functions() == sorted(N.exported_symbols())


def test_library_loads_and_exports_every_symbol():
    lib = N.load()
    for name in header_functions():
        assert hasattr(lib, name), name
        assert ctypes.cast(getattr(lib, name), ctypes.c_void_p).value
    assert lib.ffx_abi_version() == 3


def test_struct_layouts_match_the_header():
    # sizes of the C structs (natural alignment, 64-bit pointers)
    assert ctypes.sizeof(N.FfxGrid) == 36
    assert ctypes.sizeof(N.FfxSolids) == 16 + 24 + 8   # solid, halo, wall[3], clear
    assert ctypes.sizeof(N.FfxSources) == 4 * (2 + 3 + 3 + 1 + 3 + 1 + 128)
    assert ctypes.sizeof(N.FfxScalarChannel) == 4 * 8 + 4 * 5 + 4
    assert ctypes.sizeof(N.FfxGraphLevel) == 12 + 4 + 8 + 8 + 12 + 4 + 8   # ..., w[3], pad, links


def test_argument_errors_are_reported_without_a_device():
    lib = N.load()
    g = N.FfxGrid(0, 4, 4, 1, 1, 1, 0, 0, 0)
    st = lib.ffx_divergence(ctypes.byref(g), None, 0, None, None, None, None, None)
    assert st == N.FFX_ERR_INVALID
    assert b'ffx_divergence' in lib.ffx_last_error()
    with pytest.raises(N.FfxError) as err:
        N.check(st)
    assert err.value.status == N.FFX_ERR_INVALID
    assert lib.ffx_direct_solve(4096, None, None, 1.0, None, None) == N.FFX_ERR_INVALID
    assert lib.ffx_divergence_stats_workspace(1 << 20) > 0


def test_grid_struct_carries_the_fp64_reciprocal_cell_size():
    g = N.grid_struct((12, 10, 8), (1.3, 0.8, 1.7))
    assert (g.nx, g.ny, g.nz) == (12, 10, 8)
    assert g.ix == pytest.approx(1 / (1.3 / 12), rel=1e-7)
    assert g.iz == pytest.approx(1 / (1.7 / 8), rel=1e-7)


def test_reference_shader_library_exports(tmp_path):
    from oracle.glsl_ref import device as G
    if not G.LIB.exists():
        pytest.skip('reference shader library not built in this checkout')
    lib = G.load()
    assert lib.glsl_ref_kernel_count() >= 30
    assert lib.glsl_ref_kernel(b'pressure_jacobi.glsl', 1) >= 0
    assert lib.glsl_ref_kernel(b'volume.frag.glsl', 0) == -1


def test_build_entry_compiles_and_loads():
    """The build entry point (nvcc for sm_100a, in place; incremental) imports
    the package and finds every bound symbol."""
    import __graft_entry__ as entry
    entry.build()
