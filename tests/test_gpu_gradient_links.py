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
