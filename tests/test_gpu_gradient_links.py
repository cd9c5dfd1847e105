"""The pressure-gradient pass with the collider test read from the level-0
link bytes (ffx_gradient_links) against the pass that tests the mask itself
(ffx_gradient): faces, the divergence after the projection and the face maxima
bit for bit, on a random collider mask with ragged tiles, in FP32 and BF16
storage, with the dilated halo mask the solvers pass (ffx_dilate_mask)."""
import ctypes as C

import pytest
import torch

from fluxfx_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('storage', ['FP32', 'BF16'])
@pytest.mark.parametrize('shape, extent', [((36, 20, 17), (1.3, 0.8, 0.7)), ((32, 32, 32), (1.0, 1.0, 1.0))])
def test_gradient_with_links_equals_mask_test(shape, extent, storage):
    lib = N.load()
    nx, ny, nz = shape
    g = torch.Generator().manual_seed(nx + ny + nz)
    mask = (torch.rand((nz, ny, nx), generator=g) < 0.2).to(torch.uint8).cuda()
    dtype, code = (torch.float32, N.FFX_F32) if storage == 'FP32' else (torch.bfloat16, N.FFX_BF16)
    faces = [torch.randn(s, generator=g).to(dtype).cuda()
             for s in ((nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx))]
    p = torch.randn((nz, ny, nx), generator=g).cuda()
    grid = N.grid_struct(shape, extent)
    halo = torch.empty_like(mask)
    N.check(lib.ffx_dilate_mask(C.byref(grid), C.c_void_p(mask.data_ptr()), C.c_void_p(halo.data_ptr()), None))
    solids = N.FfxSolids(mask.data_ptr(), halo.data_ptr(), (C.c_void_p * 3)())
    level = N.FfxGraphLevel(nx, ny, nz, None, mask.data_ptr(), (N.f32 * 3)(1.0, 1.0, 1.0), 1.0, None)
    links = torch.empty((nz, ny, nx), dtype=torch.uint8, device='cuda')
    N.check(lib.ffx_graph_links(C.byref(level), C.c_void_p(links.data_ptr()), None))
    outs = []
    for use_links in (False, True):
        o = [torch.full_like(f, 7.0) for f in faces]
        div = torch.full((nz, ny, nx), 7.0, device='cuda')
        mx = torch.zeros(3, device='cuda')
        args = [C.byref(grid), C.byref(solids), code, *[C.c_void_p(f.data_ptr()) for f in faces],
                C.c_void_p(p.data_ptr()), 0.37, *[C.c_void_p(x.data_ptr()) for x in o], C.c_void_p(div.data_ptr()),
                C.c_void_p(mx.data_ptr())]
        if use_links:
            N.check(lib.ffx_gradient_links(*args, C.c_void_p(links.data_ptr()), None))
        else:
            N.check(lib.ffx_gradient(*args, None))
        torch.cuda.synchronize()
        outs.append(o + [div, mx])
    for a, b in zip(*outs):
        assert torch.equal(a, b)


@pytest.mark.parametrize('storage', ['FP32', 'BF16'])
def test_unrounded_divergence_output(storage):
    """ffx_gradient_ex also writes the divergence of the corrected faces before
    they are rounded to storage: equal to div_after in FP32 storage; in BF16
    storage the divergence of the FP32 result, which the rounding perturbs by
    about 2^-9 of the face values."""
    lib = N.load()
    nx, ny, nz = 40, 24, 20
    shape, extent = (nx, ny, nz), (1.0, 0.6, 0.5)
    g = torch.Generator().manual_seed(5)
    dtype, code = (torch.float32, N.FFX_F32) if storage == 'FP32' else (torch.bfloat16, N.FFX_BF16)
    faces = [torch.randn(s, generator=g).to(dtype).cuda()
             for s in ((nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx))]
    p = torch.randn((nz, ny, nx), generator=g).cuda()
    grid = N.grid_struct(shape, extent)
    o = [torch.empty_like(f) for f in faces]
    div = torch.empty((nz, ny, nx), device='cuda')
    div32 = torch.empty((nz, ny, nx), device='cuda')
    mx = torch.zeros(3, device='cuda')
    N.check(lib.ffx_gradient_ex(C.byref(grid), None, code, *[C.c_void_p(f.data_ptr()) for f in faces],
                                C.c_void_p(p.data_ptr()), 0.37, *[C.c_void_p(x.data_ptr()) for x in o],
                                C.c_void_p(div.data_ptr()), C.c_void_p(mx.data_ptr()), None,
                                C.c_void_p(div32.data_ptr()), None))
    ref = [torch.empty_like(f) for f in faces]
    div_ref = torch.empty_like(div)
    N.check(lib.ffx_gradient(C.byref(grid), None, code, *[C.c_void_p(f.data_ptr()) for f in faces],
                             C.c_void_p(p.data_ptr()), 0.37, *[C.c_void_p(x.data_ptr()) for x in ref],
                             C.c_void_p(div_ref.data_ptr()), None, None))
    torch.cuda.synchronize()
    for a, b in zip(o, ref):
        assert torch.equal(a, b)
    assert torch.equal(div, div_ref)
    if storage == 'FP32':
        assert torch.equal(div32, div)
    else:
        # FP64 divergence of the unrounded faces, recomputed on the host
        inv = [n / e for n, e in zip(shape, extent)]
        f32 = [f.double() for f in faces]
        pd = p.double()
        gx = torch.zeros_like(f32[0]); gx[:, :, 1:-1] = (pd[:, :, 1:] - pd[:, :, :-1]) * inv[0]
        gy = torch.zeros_like(f32[1]); gy[:, 1:-1, :] = (pd[:, 1:, :] - pd[:, :-1, :]) * inv[1]
        gz = torch.zeros_like(f32[2]); gz[1:-1, :, :] = (pd[1:, :, :] - pd[:-1, :, :]) * inv[2]
        u = f32[0] - 0.37 * gx; u[:, :, 0] = 0; u[:, :, -1] = 0
        v = f32[1] - 0.37 * gy; v[:, 0, :] = 0; v[:, -1, :] = 0
        w = f32[2] - 0.37 * gz; w[0] = 0; w[-1] = 0
        exact = (u[:, :, 1:] - u[:, :, :-1]) * inv[0] + (v[:, 1:, :] - v[:, :-1, :]) * inv[1] + \
            (w[1:] - w[:-1]) * inv[2]
        scale = float(exact.abs().max())
        assert float((div32.double() - exact).abs().max()) <= 1e-5 * scale
        assert float((div.double() - exact).abs().max()) > 1e-4 * scale     # the stored faces are rounded
