"""ctypes binding of ``libffx_core.so`` (declared in ``include/ffx.h``).

The library is loaded from ``fluxfx_b200/_lib`` (built in place by
``python -m fluxfx_b200.build``). There is no fallback: if the library is
missing, every solver constructor raises ``NativeUnavailable``.
"""
import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / '_lib' / 'libffx_core.so'

FFX_OK, FFX_ERR_INVALID, FFX_ERR_LAUNCH, FFX_ERR_NOT_CONVERGED, FFX_ERR_TIMEOUT, FFX_ERR_CUDA = range(6)
FFX_F32, FFX_BF16 = 0, 1
FFX_PACK_U8 = 2
STATUS_NAMES = {0: 'OK', 1: 'INVALID', 2: 'LAUNCH', 3: 'NOT_CONVERGED', 4: 'TIMEOUT', 5: 'CUDA'}

vp = C.c_void_p
i32 = C.c_int32
f32 = C.c_float
i64 = C.c_int64
f3 = f32 * 3
n3 = i32 * 3


class NativeUnavailable(RuntimeError):
    """libffx_core.so could not be loaded (not built, or no CUDA driver)."""


class FfxError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class FfxGrid(C.Structure):
    _fields_ = [('nx', i32), ('ny', i32), ('nz', i32), ('ex', f32), ('ey', f32), ('ez', f32),
                ('ix', f32), ('iy', f32), ('iz', f32)]


class FfxSolids(C.Structure):
    _fields_ = [('solid', vp), ('halo', vp), ('wall', vp * 3), ('clear', vp)]


class FfxSources(C.Structure):
    _fields_ = [('count', i32), ('single_solid_profile', i32), ('single_center', f3), ('single_start', f3),
                ('single_radius', f32), ('single_jet', f3), ('single_coupling', f32), ('table', f32 * 128)]


class FfxDeviceInfo(C.Structure):
    _fields_ = [('device', i32), ('sm_count', i32), ('cc_major', i32), ('cc_minor', i32),
                ('total_bytes', i64), ('name', C.c_char * 128)]


class FfxScalarChannel(C.Structure):
    _fields_ = [('field', vp), ('predictor', vp), ('reverse', vp), ('out', vp), ('rate', f32), ('decay', f32),
                ('target', f32), ('channel', i32), ('table_target', i32)]


class FfxGraphLevel(C.Structure):
    _fields_ = [('nx', i32), ('ny', i32), ('nz', i32), ('edges', vp), ('solid', vp), ('w', f3),
                ('coarse_scale', f32), ('links', vp)]


TAIL_LEVELS = 8
MOVING_MAX = 8


class FfxTailLevel(C.Structure):
    _fields_ = [('level', FfxGraphLevel), ('p', vp), ('q', vp), ('rhs', vp)]


class FfxGraphTail(C.Structure):
    _fields_ = [('count', i32), ('pre', i32), ('post', i32), ('omega', f32), ('inverse', vp),
                ('levels', FfxTailLevel * TAIL_LEVELS)]


class FfxBrickStats(C.Structure):
    _fields_ = [("capacity", C.c_uint32), ("active", C.c_uint32), ("metadata_bytes", C.c_uint64)]


class FfxArenaStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("capacity", "used", "peak", "allocations", "live", "largest_free")]


class FfxSparseLevel(C.Structure):
    _fields_ = [("n", C.c_int32), ("side", C.c_int32), ("mode", C.c_int32), ("sparse", C.c_int32),
                ("map", C.c_void_p), ("active", C.c_void_p), ("coords", C.c_void_p), ("count", C.c_int32)]


class FfxTensorView(C.Structure):
    _fields_ = [('data', vp), ('pitch', i32), ('offset', i32)]


class FfxConv(C.Structure):
    _fields_ = [('batch', i32), ('in_dims', i32 * 3), ('out_dims', i32 * 3), ('c1', i32), ('c2', i32),
                ('cout', i32), ('ksize', i32), ('stride', i32), ('pad', i32), ('transposed', i32),
                ('in1', FfxTensorView), ('in2', FfxTensorView), ('weight', vp), ('bias', vp), ('relu', i32),
                ('accumulate', i32), ('out', vp), ('out_pitch', i32), ('out_offset', i32), ('out_f32', vp),
                ('out_f32_pitch', i32)]


BATCH_MAX = 64
BATCH_LEVELS = 8
(PASS_PREDICTOR, PASS_VELOCITY, PASS_DIVERGENCE, PASS_SCALE, PASS_GRADIENT, PASS_SCALAR_PREDICTOR,
 PASS_SCALAR_REVERSE, PASS_SCALAR_FINAL, PASS_RESIDUAL_MAX, PASS_SMOOTH, PASS_RESIDUAL_RESTRICT, PASS_PROLONG_SMOOTH,
 PASS_DIRECT, PASS_L0_SMOOTH, PASS_L0_PROLONG_SMOOTH, PASS_L0_RESIDUAL_RESTRICT, PASS_L0_RESIDUAL_MAX,
 PASS_KINDS) = range(18)
PASS_NAMES = ('predictor', 'velocity', 'divergence', 'scale', 'gradient', 'scalar_predictor', 'scalar_reverse',
              'scalar_final', 'residual_max', 'smooth', 'residual_restrict', 'prolong_smooth', 'direct',
              'l0_smooth', 'l0_prolong_smooth', 'l0_residual_restrict', 'l0_residual_max')
# pass kinds with a fixed tile (the level-0 four-cell kernels' 32 x 8 block): only the grid is tuned
FIXED_TILE_PASSES = (PASS_L0_SMOOTH, PASS_L0_PROLONG_SMOOTH, PASS_L0_RESIDUAL_RESTRICT, PASS_L0_RESIDUAL_MAX)


class FfxBatchLevel(C.Structure):
    _fields_ = [('level', FfxGraphLevel), ('p', vp), ('q', vp), ('rhs', vp)]


class FfxBatchDomain(C.Structure):
    _fields_ = [('grid', FfxGrid), ('solid', vp), ('halo', vp), ('u', vp), ('v', vp), ('w', vp), ('pu', vp),
                ('pv', vp), ('pw', vp), ('bu', vp), ('bv', vp), ('bw', vp), ('density', vp * 2),
                ('temperature', vp * 2), ('predictor', vp * 2), ('reverse', vp * 2), ('after', vp),
                ('sources', FfxSources), ('velocity_corrected', i32), ('scalar_corrected', i32), ('blend', f32),
                ('lift', f32), ('weight', f32), ('density_channel', FfxScalarChannel),
                ('heat_channel', FfxScalarChannel), ('cell', C.c_double), ('cfl', C.c_double),
                ('dt_max', C.c_double), ('dt0', f32), ('levels', i32), ('level', FfxBatchLevel * BATCH_LEVELS),
                ('tail_start', i32), ('inverse', vp), ('pre', i32), ('post', i32), ('max_cycles', i32),
                ('warm_start', i32), ('tolerance', C.c_double), ('face_trace', vp * 3), ('cell_trace', vp),
                ('clear', vp), ('cell_ok', vp)]


class FfxBatchStats(C.Structure):
    _fields_ = [('dt', f32), ('last_dt', f32), ('last_cycles', i32), ('total_cycles', i32), ('steps', i32),
                ('maxima', f3), ('time', C.c_double), ('loop_iterations', i64)]


P = C.POINTER
_PROTOTYPES = {
    'ffx_abi_version': (C.c_int, []),
    'ffx_last_error': (C.c_char_p, []),
    'ffx_device_info': (C.c_int, [C.c_int, P(FfxDeviceInfo)]),
    'ffx_probe_3d': (C.c_int, [vp, vp]),
    'ffx_seed_scalar': (C.c_int, [P(FfxGrid), C.c_int, f3, f32, f32, vp, vp]),
    'ffx_seed_faces': (C.c_int, [P(FfxGrid), C.c_int, f3, f32, vp, vp, vp, vp]),
    'ffx_raster_colliders': (C.c_int, [P(FfxGrid), C.c_double * 3, C.c_int, vp, vp, vp]),
    'ffx_dilate_mask': (C.c_int, [P(FfxGrid), vp, vp, vp]),
    'ffx_clearance': (C.c_int, [P(FfxGrid), vp, vp, vp]),
    'ffx_halo_clearance': (C.c_int, [P(FfxGrid), vp, vp, vp, vp]),
    'ffx_division_mismatches': (C.c_int, [f32, vp, vp]),
    'ffx_solid_clear': (C.c_int, [P(FfxGrid), C.c_int, vp, vp, vp, vp]),
    'ffx_face_predictor': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, f32, vp, vp, vp, vp]),
    'ffx_set_transport_tiling': (C.c_int, [C.c_int]),
    'ffx_set_edge_streaming': (C.c_int, [C.c_int]),
    'ffx_set_dependent_launch': (C.c_int, [C.c_int]),
    'ffx_pack_channels': (C.c_int, [i64, C.c_int, P(vp), P(C.c_int), vp, vp]),
    'ffx_loop_begin': (C.c_int, [vp, P(vp)]),
    'ffx_loop_decide': (C.c_int, [vp, vp, vp, C.c_double, C.c_int32, vp, vp]),
    'ffx_loop_reset_counter': (C.c_int, [vp, vp]),
    'ffx_zero_if_unscaled': (C.c_int, [vp, vp, i64, vp]),
    'ffx_loop_while': (C.c_int, [vp, P(vp)]),
    'ffx_loop_end_while': (C.c_int, [vp]),
    'ffx_loop_end': (C.c_int, [vp]),
    'ffx_loop_launch': (C.c_int, [vp, vp]),
    'ffx_loop_destroy': (C.c_int, [vp]),
    'ffx_face_predictor_trace': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, f32, vp, vp, vp, P(vp),
                                           vp]),
    'ffx_advect_velocity': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, vp, vp, vp, f32, C.c_int, f32,
                                      P(FfxSources), vp, vp, f32, f32, C.c_int, vp, vp, vp, vp]),
    'ffx_advect_velocity_trace': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, vp, vp, vp, f32, C.c_int,
                                            f32, P(FfxSources), vp, vp, f32, f32, C.c_int, vp, vp, vp, P(vp), vp]),
    'ffx_mac_advect_velocity': (C.c_int, [P(FfxGrid), C.c_int, vp, vp, vp, f32, vp, vp, vp, vp]),
    'ffx_buoyancy': (C.c_int, [P(FfxGrid), C.c_int, vp, vp, vp, f32, f32, f32, vp, vp]),
    'ffx_scalar_transport': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, f32, C.c_int, P(vp), P(vp), vp]),
    'ffx_scalar_transport_trace': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, f32, C.c_int, P(vp),
                                             P(vp), vp, vp]),
    'ffx_advect_scalars': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, f32, C.c_int, P(FfxSources),
                                     C.c_int, P(FfxScalarChannel), vp, vp]),
    'ffx_advect_scalars_trace': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, f32, C.c_int,
                                           P(FfxSources), C.c_int, P(FfxScalarChannel), vp, vp, vp]),
    # the same passes with the time step read on the device (a float pointer in place of dt)
    'ffx_face_predictor_dt': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, vp, vp, vp, vp, P(vp), vp]),
    'ffx_advect_velocity_dt': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, vp, vp, vp, vp, C.c_int,
                                         f32, P(FfxSources), vp, vp, f32, f32, C.c_int, vp, vp, vp, P(vp), vp]),
    'ffx_scalar_transport_dt': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, vp, f32, C.c_int, P(vp),
                                          P(vp), vp, vp]),
    'ffx_advect_scalars_dt': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, vp, C.c_int,
                                        P(FfxSources), C.c_int, P(FfxScalarChannel), vp, vp, vp]),
    'ffx_scalar_reverse_ok': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, C.c_float, vp, C.c_int,
                                        vp, vp, vp, vp, vp]),
    'ffx_advect_scalars_ok': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, C.c_float, vp, C.c_int,
                                        P(FfxSources), C.c_int, P(FfxScalarChannel), vp, vp, vp, vp]),
    'ffx_next_dt': (C.c_int, [vp, vp, vp, C.c_double, C.c_double, C.c_double, vp]),
    'ffx_add': (C.c_int, [i64, vp, vp, vp, vp]),
    'ffx_bricks_create': (C.c_int, [C.c_uint32, P(vp)]),
    'ffx_bricks_destroy': (C.c_int, [vp]),
    'ffx_bricks_lookup': (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32, P(C.c_int32)]),
    'ffx_bricks_activate': (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32, P(C.c_int32)]),
    'ffx_bricks_deactivate': (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32, P(C.c_int32)]),
    'ffx_bricks_neighbors': (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32, P(C.c_int32)]),
    'ffx_bricks_activate_box': (C.c_int, [vp, P(C.c_int32), P(C.c_int32)]),
    'ffx_bricks_stats': (C.c_int, [vp, P(FfxBrickStats)]),
    'ffx_bricks_active': (C.c_int, [vp, P(C.c_int32), P(C.c_int32), C.c_uint32]),
    'ffx_arena_create': (C.c_int, [C.c_uint64, P(vp)]),
    'ffx_arena_destroy': (C.c_int, [vp]),
    'ffx_arena_allocate': (C.c_int, [vp, C.c_uint64, P(C.c_uint64)]),
    'ffx_arena_get': (C.c_int, [vp, C.c_uint64, P(C.c_uint64), P(C.c_uint64), P(C.c_uint64)]),
    'ffx_arena_release': (C.c_int, [vp, C.c_uint64]),
    'ffx_arena_stats': (C.c_int, [vp, P(FfxArenaStats)]),
    'ffx_sparse_divergence': (C.c_int, [P(FfxSparseLevel), vp, C.c_int32, vp, vp]),
    'ffx_sparse_jacobi': (C.c_int, [P(FfxSparseLevel), vp, vp, vp, vp]),
    'ffx_sparse_residual': (C.c_int, [P(FfxSparseLevel), vp, vp, vp, vp]),
    'ffx_sparse_gradient': (C.c_int, [P(FfxSparseLevel), vp, vp, C.c_int32, vp, vp]),
    'ffx_sparse_restrict': (C.c_int, [P(FfxSparseLevel), vp, P(FfxSparseLevel), vp, vp]),
    'ffx_sparse_prolong': (C.c_int, [P(FfxSparseLevel), vp, P(FfxSparseLevel), vp, vp]),
    'ffx_gradient_ex': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, vp, f32, vp, vp, vp, vp, vp, vp, vp,
                                  vp]),
    'ffx_scale_by_ratio': (C.c_int, [i64, vp, vp, vp]),
    'ffx_extrapolate_pressure': (C.c_int, [i64, vp, vp, vp, C.c_float, C.c_int32, vp]),
    'ffx_extrapolate_pressure2': (C.c_int, [i64, vp, vp, vp, vp, vp, vp, C.c_float, C.c_int32, vp]),
    'ffx_advect_open': (C.c_int, [P(FfxGrid), C.c_int, vp, f32, f3, f32, f3, f32, f32, f32, vp, vp]),
    'ffx_mac_advect_density': (C.c_int, [P(FfxGrid), C.c_int, vp, vp, vp, vp, f32, f3, f32, f32, f32, vp, vp]),
    'ffx_walls': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, vp, vp, vp, vp]),
    'ffx_divergence': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, vp, vp]),
    'ffx_walls_divergence': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, vp, vp, vp, vp, vp]),
    'ffx_gradient': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, vp, f32, vp, vp, vp, vp, vp, vp]),
    'ffx_gradient_links': (C.c_int, [P(FfxGrid), P(FfxSolids), C.c_int, vp, vp, vp, vp, f32, vp, vp, vp, vp, vp, vp,
                                     vp]),
    'ffx_jacobi': (C.c_int, [n3, f3, vp, vp, vp, f32, f32, vp, vp]),
    'ffx_scale': (C.c_int, [i64, vp, f32, vp, vp]),
    'ffx_mg_residual': (C.c_int, [n3, f3, vp, vp, f32, vp, vp]),
    'ffx_mg_restrict': (C.c_int, [n3, vp, vp, vp]),
    'ffx_mg_residual_restrict': (C.c_int, [n3, f3, vp, vp, f32, vp, vp]),
    'ffx_mg_prolong': (C.c_int, [n3, vp, vp, vp, vp]),
    'ffx_direct_solve': (C.c_int, [i32, vp, vp, f32, vp, vp]),
    'ffx_mg_residual_max': (C.c_int, [n3, f3, vp, vp, f32, vp, vp]),
    'ffx_graph_smooth': (C.c_int, [P(FfxGraphLevel), vp, vp, f32, vp, vp]),
    'ffx_graph_smooth2': (C.c_int, [P(FfxGraphLevel), vp, vp, f32, vp, vp, vp]),
    'ffx_graph_residual_max_smooth': (C.c_int, [P(FfxGraphLevel), vp, vp, f32, vp, vp, vp]),
    'ffx_graph_prolong_smooth2': (C.c_int, [P(FfxGraphLevel), vp, vp, vp, f32, vp, vp, vp]),
    'ffx_graph_residual': (C.c_int, [P(FfxGraphLevel), vp, vp, vp, vp]),
    'ffx_graph_residual_restrict': (C.c_int, [P(FfxGraphLevel), vp, vp, vp, vp]),
    'ffx_graph_residual_restrict_zero': (C.c_int, [P(FfxGraphLevel), vp, vp, vp, vp, vp]),
    'ffx_graph_prolong': (C.c_int, [P(FfxGraphLevel), vp, vp, vp, vp]),
    'ffx_graph_prolong_smooth': (C.c_int, [P(FfxGraphLevel), vp, vp, vp, f32, vp, vp]),
    'ffx_graph_residual_max': (C.c_int, [P(FfxGraphLevel), vp, vp, vp, vp]),
    'ffx_graph_coarsen': (C.c_int, [P(FfxGraphLevel), vp, vp, vp]),
    'ffx_graph_level0_edges': (C.c_int, [P(FfxGraphLevel), vp, vp]),
    'ffx_graph_links': (C.c_int, [P(FfxGraphLevel), vp, vp]),
    'ffx_graph_tail': (C.c_int, [P(FfxGraphTail), vp]),
    'ffx_conv_forward': (C.c_int, [P(FfxConv), vp]),
    'ffx_conv_forward_tc': (C.c_int, [P(FfxConv), vp]),
    'ffx_conv_timeouts': (C.c_int, [P(i32), i32]),
    'ffx_conv_packed_bytes': (C.c_int, [P(FfxConv), P(i64)]),
    'ffx_conv_pack_weights': (C.c_int, [P(FfxConv), vp, vp]),
    'ffx_conv_forward_tma': (C.c_int, [P(FfxConv), vp, vp]),
    'ffx_conv_weight_grad': (C.c_int, [P(FfxConv), vp, i32, vp, vp]),
    'ffx_relu_backward': (C.c_int, [i64, i32, vp, i32, vp, i32, i32, vp]),
    'ffx_bias_grad': (C.c_int, [i64, i32, vp, i32, vp, vp]),
    'ffx_weight_transpose': (C.c_int, [i32, i32, i32, i32, vp, vp, vp]),
    'ffx_adam': (C.c_int, [i64, vp, vp, vp, vp, vp, f32, f32, f32, f32, i32, vp]),
    'ffx_pack_input': (C.c_int, [i64, vp, vp, f32, vp, vp]),
    'ffx_mse_grad': (C.c_int, [i64, vp, i32, vp, vp, f32, vp, vp, vp]),
    'ffx_unpack_channel': (C.c_int, [i64, vp, i32, f32, vp, vp]),
    'ffx_unpack_channel_scaled': (C.c_int, [i64, vp, i32, vp, C.c_double, vp, vp]),
    'ffx_pack_input_scaled': (C.c_int, [i64, vp, vp, vp, vp, vp]),
    'ffx_mask_restrict': (C.c_int, [n3, vp, i32, vp, vp]),
    'ffx_curl': (C.c_int, [P(FfxGrid), C.c_int, vp, vp, vp, vp, vp]),
    'ffx_confine': (C.c_int, [P(FfxGrid), C.c_int, vp, vp, vp, vp, f32, f32, f32, vp, vp, vp, vp]),
    'ffx_combustion': (C.c_int, [P(FfxGrid), C.c_int, vp, vp, vp, f32, f32, f32, f32, f32, vp, vp, vp, vp, vp]),
    'ffx_moving_mask': (C.c_int, [P(FfxGrid), C.c_int, vp, vp, vp, vp]),
    'ffx_moving_walls': (C.c_int, [P(FfxGrid), vp, C.c_int, vp, vp, vp, vp, vp]),
    'ffx_moving_remap': (C.c_int, [P(FfxGrid), C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    'ffx_graph_smooth_zero': (C.c_int, [P(FfxGraphLevel), vp, f32, vp, vp]),
    'ffx_graph_smooth_dot': (C.c_int, [P(FfxGraphLevel), vp, vp, f32, vp, vp, C.c_double, vp]),
    'ffx_graph_prolong_smooth_dot': (C.c_int, [P(FfxGraphLevel), vp, vp, vp, f32, vp, vp, C.c_double, vp]),
    'ffx_pcg_direction_apply': (C.c_int, [P(FfxGraphLevel), vp, vp, vp, vp, vp, vp, vp, vp]),
    'ffx_pcg_update': (C.c_int, [i64, vp, vp, vp, vp, vp, vp, vp, vp]),
    'ffx_dot': (C.c_int, [i64, vp, vp, C.c_double, vp, vp]),
    'ffx_max_abs': (C.c_int, [i64, C.c_int, vp, vp, vp]),
    'ffx_divergence_stats_workspace': (C.c_size_t, [i64]),
    'ffx_divergence_stats': (C.c_int, [i64, vp, vp, vp, vp, C.c_size_t, vp]),
    'ffx_divergence_stats_static': (C.c_int, [i64, vp, vp, vp, vp]),
    'ffx_batch_workspace_bytes': (C.c_int, [P(FfxBatchDomain), i32, P(i64)]),
    'ffx_batch_create': (C.c_int, [P(FfxBatchDomain), i32, vp, i64, P(vp)]),
    'ffx_batch_set_config': (C.c_int, [vp, i32, i32, i32]),
    'ffx_batch_tune_pass': (C.c_int, [vp, i32, vp]),
    'ffx_batch_graph': (C.c_int, [vp, i32, P(vp)]),
    'ffx_batch_launch': (C.c_int, [vp, vp, i32, vp]),
    'ffx_batch_graph_free': (C.c_int, [vp]),
    'ffx_batch_stats': (C.c_int, [vp, P(FfxBatchStats), vp]),
    'ffx_batch_parity': (C.c_int, [vp]),
    'ffx_batch_destroy': (C.c_int, [vp]),
}

_LIB = None


def exported_symbols():
    return tuple(_PROTOTYPES)


def load(path=None):
    """Load the library once and attach argument/return types."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    target = Path(path) if path else Path(os.environ.get('FFX_CORE_LIB', LIB_PATH))
    if not target.exists():
        raise NativeUnavailable(f"{target} is missing; build it with `python -m fluxfx_b200.build`")
    try:
        lib = C.CDLL(str(target))
    except OSError as exc:
        raise NativeUnavailable(f"cannot load {target}: {exc}") from exc
    for name, (res, args) in _PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.ffx_abi_version() != 3:
        raise NativeUnavailable("libffx_core ABI version mismatch")
    if path is None:
        _LIB = lib
    return lib


def check(status):
    if status != FFX_OK:
        msg = load().ffx_last_error()
        raise FfxError(status, msg.decode() if msg else '')


def call(name, *args):
    """Invoke an entry point and raise FfxError on a non-OK status."""
    check(getattr(load(), name)(*args))


def grid_struct(shape, extent):
    """FfxGrid for a cell shape (nx, ny, nz) and an FP64 extent."""
    nx, ny, nz = shape
    inv = [1.0 / (e / n) for e, n in zip(extent, shape)]
    return FfxGrid(nx, ny, nz, *[float(e) for e in extent], *inv)


def face_starts_match(shape, extent):
    """True when the face predictor's start point (x + o) h and the velocity
    correction's (x + o) e / n (times 1/n on power-of-two grids) are the same
    FP32 value for every face coordinate x + o (o = 0, 1/2) of every axis --
    the library's own test (ffx_common.cuh, face_starts_match) in NumPy FP32.
    The correction then reuses the predictor's face departure points."""
    import numpy as np
    p2 = grid_pow2(shape, extent)
    for n, e in zip(shape, extent):
        e32, n32 = np.float32(e), np.float32(n)
        h32 = np.float32(e32 / n32)
        x = (np.arange(n + 1, dtype=np.float32)[:, None] + np.array([0.0, 0.5], dtype=np.float32)).ravel()
        a = x * h32
        xe = x * e32
        b = xe * np.float32(np.float32(1.0) / n32) if p2 else xe / n32
        if not np.array_equal(a, b):
            return False
    return True


def grid_pow2(shape, extent):
    """True when every FP32 extent, cell count and spacing (extent / count in
    FP32) is a power of two: the kernels then divide by exact reciprocals and
    the two transport passes form the same start points."""
    import math

    import numpy as np

    def pow2(v):
        v = float(v)
        return v > 0 and math.frexp(v)[0] == 0.5
    for n, e in zip(shape, extent):
        e32 = np.float32(e)
        h32 = np.float32(e32 / np.float32(n))
        if not (pow2(e32) and pow2(n) and pow2(h32)):
            return False
    return True
