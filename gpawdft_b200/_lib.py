"""ctypes binding of the C ABI in include/gpwgrid.h (libgpwgrid.so).

This is the same binding a reference-side maintainer would add to call the
library from GPAW's Python layer.  Loading fails loudly: there is no CPU
fallback for any entry point.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libgpwgrid.so')

GPW_OK = 0
GPW_ENOMEM = 12
GPW_EINVAL = 22
GPW_ENOTSUP = 95
GPW_ETIMEDOUT = 110
GPW_ECONV = 1001
GPW_ECUDA = 1002

GPW_F64, GPW_C128, GPW_F32, GPW_C64 = 0, 1, 2, 3

# every symbol include/gpwgrid.h declares
EXPORTS = [
    'gpw_last_error', 'gpw_version',
    'gpw_operator_new', 'gpw_operator_apply', 'gpw_operator_apply_potential',
    'gpw_operator_apply_fused',
    'gpw_operator_relax',
    'gpw_operator_get_diagonal_element', 'gpw_operator_residual',
    'gpw_operator_residual_noalloc', 'gpw_operator_free',
    'gpw_woperator_new', 'gpw_woperator_apply', 'gpw_woperator_relax',
    'gpw_woperator_get_diagonal_element', 'gpw_woperator_free',
    'gpw_transformer_new', 'gpw_transformer_apply', 'gpw_transformer_free',
    'gpw_transformer_apply_subtract',
    'gpw_axpy', 'gpw_scal', 'gpw_sum', 'gpw_dot', 'gpw_dotc_pairs',
    'gpw_copy_box', 'gpw_mul', 'gpw_tune_export', 'gpw_tune_import',
    'gpw_add_scalar',
    'gpw_poisson_charge_prepare', 'gpw_poisson_charge_finish',
    'gpw_poisson_new', 'gpw_poisson_solve', 'gpw_poisson_last_stats',
    'gpw_poisson_solve_async', 'gpw_poisson_collect',
    'gpw_poisson_time_level0', 'gpw_poisson_set_inner_schedule',
    'gpw_set_tma_variant', 'gpw_set_bloch_layout', 'gpw_bloch_launch_count',
    'gpw_set_restrict_layout', 'gpw_restrict_rows_launch_count',
    'gpw_poisson_set_device_loop', 'gpw_set_pdl', 'gpw_poisson_set_cluster',
    'gpw_poisson_set_fusion',
    'gpw_poisson_solve_many', 'gpw_poisson_last_latency',
    'gpw_poisson_profile_iteration', 'gpw_poisson_free',
    'gpw_nn_conv3', 'gpw_nn_wgrad_scratch', 'gpw_nn_conv3_wgrad',
    'gpw_nn_flip_weights', 'gpw_nn_gelu_backward', 'gpw_nn_pool2',
    'gpw_nn_pool2_backward', 'gpw_nn_upsample2_add',
    'gpw_nn_upsample2_backward', 'gpw_nn_head', 'gpw_nn_head_backward',
    'gpw_nn_partials', 'gpw_nn_pack_input', 'gpw_nn_upsample_add_f32',
    'gpw_nn_downsum_f32', 'gpw_nn_mse', 'gpw_nn_unpack_output', 'gpw_nn_adam',
    'gpw_nn_gaussians', 'gpw_nn_channel_sum',
]

_c_i64p = ctypes.POINTER(ctypes.c_int64)
_c_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

_SIGS = {
    'gpw_last_error': (ctypes.c_char_p, []),
    'gpw_version': (ctypes.c_char_p, []),
    'gpw_operator_new': (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp,
                                        ctypes.c_int, _vp, ctypes.c_int,
                                        ctypes.c_int, ctypes.POINTER(_vp)]),
    'gpw_operator_apply': (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp,
                                          ctypes.c_int64, _vp, _vp]),
    'gpw_operator_apply_potential': (ctypes.c_int, [_vp, ctypes.c_int, _vp,
                                                    _vp, ctypes.c_int64, _vp,
                                                    _vp, _vp]),
    'gpw_operator_apply_fused': (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp,
                                                ctypes.c_int64, _vp, _vp, _vp,
                                                ctypes.c_double, _vp]),
    'gpw_operator_relax': (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int,
                                          _vp, _vp, ctypes.c_int64,
                                          ctypes.c_int, ctypes.c_double,
                                          _vp]),
    'gpw_operator_get_diagonal_element': (ctypes.c_int, [_vp, _c_dp]),
    'gpw_operator_residual': (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp,
                                             ctypes.c_int64, _vp, _vp]),
    'gpw_operator_residual_noalloc': (ctypes.c_int, [_vp, ctypes.c_int, _vp,
                                                     _vp, _vp, ctypes.c_int64,
                                                     _vp, _vp]),
    'gpw_operator_free': (None, [_vp]),
    'gpw_woperator_new': (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp,
                                         ctypes.c_int, _vp, ctypes.c_int,
                                         ctypes.c_int, ctypes.POINTER(_vp)]),
    'gpw_woperator_apply': (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp,
                                           ctypes.c_int64, _vp, _vp]),
    'gpw_woperator_relax': (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp,
                                           ctypes.c_int, ctypes.c_double,
                                           _vp]),
    'gpw_woperator_get_diagonal_element': (ctypes.c_int, [_vp, _vp, _c_dp,
                                                          _vp]),
    'gpw_woperator_free': (None, [_vp]),
    'gpw_transformer_new': (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, _vp,
                                           _vp, _vp, ctypes.c_int,
                                           ctypes.c_int, ctypes.POINTER(_vp)]),
    'gpw_transformer_apply': (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp,
                                             ctypes.c_int64, _vp, _vp]),
    'gpw_transformer_free': (None, [_vp]),
    'gpw_transformer_apply_subtract': (ctypes.c_int, [_vp, ctypes.c_int, _vp,
                                                      _vp, _vp, ctypes.c_int64,
                                                      _vp, _vp]),
    'gpw_axpy': (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, ctypes.c_double,
                                ctypes.c_double, _vp, _vp, _vp]),
    'gpw_scal': (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, ctypes.c_double,
                                ctypes.c_double, _vp, _vp]),
    'gpw_sum': (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, ctypes.c_int64,
                               _vp, _vp, _vp]),
    'gpw_dot': (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, ctypes.c_int64,
                               _vp, _vp, _vp, _vp]),
    'gpw_copy_box': (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp,
                                    _vp, _vp, _vp]),
    'gpw_tune_export': (ctypes.c_int, [_vp, ctypes.c_int64, _c_i64p]),
    'gpw_tune_import': (ctypes.c_int, [ctypes.c_char_p,
                                       ctypes.POINTER(ctypes.c_int)]),
    'gpw_mul': (ctypes.c_int, [ctypes.c_int64, _vp, _vp, _vp, _vp]),
    'gpw_dotc_pairs': (ctypes.c_int, [ctypes.c_int, ctypes.c_int64,
                                      ctypes.c_int64, ctypes.c_int64, _vp,
                                      _vp, _vp, _vp]),
    'gpw_add_scalar': (ctypes.c_int, [ctypes.c_int, ctypes.c_int64,
                                      ctypes.c_double, _vp, _vp, _vp]),
    'gpw_poisson_charge_prepare': (ctypes.c_int, [
        ctypes.c_int64, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp,
        ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
        ctypes.c_int, _vp, _vp]),
    'gpw_poisson_charge_finish': (ctypes.c_int, [
        ctypes.c_int64, ctypes.c_int64, _vp, _vp, _vp, _vp]),
    'gpw_poisson_new': (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp,
                                       _vp, ctypes.c_int, ctypes.c_double,
                                       ctypes.c_int64, ctypes.POINTER(_vp)]),
    'gpw_poisson_solve': (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int64, _vp,
                                         ctypes.c_int, ctypes.c_int, _vp, _vp,
                                         _vp]),
    'gpw_poisson_last_stats': (ctypes.c_int, [_vp, _vp, _vp]),
    'gpw_poisson_solve_async': (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int64, _vp,
                                               ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               _vp]),
    'gpw_poisson_collect': (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, _vp, _vp]),
    'gpw_set_tma_variant': (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    'gpw_set_bloch_layout': (ctypes.c_int, [ctypes.c_int]),
    'gpw_poisson_set_device_loop': (ctypes.c_int, [_vp, ctypes.c_int]),
    'gpw_set_pdl': (ctypes.c_int, [ctypes.c_int]),
    'gpw_poisson_set_cluster': (ctypes.c_int, [_vp, ctypes.c_int]),
    'gpw_poisson_set_fusion': (ctypes.c_int, [_vp, ctypes.c_int]),
    'gpw_bloch_launch_count': (ctypes.c_int64, []),
    'gpw_set_restrict_layout': (ctypes.c_int, [ctypes.c_int]),
    'gpw_restrict_rows_launch_count': (ctypes.c_int64, []),
    'gpw_poisson_time_level0': (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int,
                                               ctypes.c_int, _vp, _vp, _vp]),
    'gpw_poisson_set_inner_schedule': (ctypes.c_int, [_vp, _vp, _vp, _vp,
                                                      ctypes.c_int]),
    'gpw_poisson_solve_many': (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp,
                                              _vp, ctypes.c_int, ctypes.c_int,
                                              _vp, _vp, _vp]),
    'gpw_poisson_last_latency': (ctypes.c_int, [_vp, ctypes.c_int64, _vp, _vp]),
    'gpw_poisson_profile_iteration': (ctypes.c_int, [_vp, ctypes.c_int64,
                                                     ctypes.c_int, ctypes.c_int,
                                                     _vp, ctypes.c_int, _vp,
                                                     ctypes.c_int, _vp, _vp]),
    'gpw_poisson_free': (None, [_vp]),
    'gpw_nn_conv3': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    'gpw_nn_wgrad_scratch': (ctypes.c_int64, [ctypes.c_int, ctypes.c_int]),
    'gpw_nn_conv3_wgrad': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    'gpw_nn_flip_weights': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    'gpw_nn_gelu_backward': (ctypes.c_int, [ctypes.c_int64, _vp, _vp, _vp, _vp]),
    'gpw_nn_pool2': (ctypes.c_int, [ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    'gpw_nn_pool2_backward': (ctypes.c_int, [ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    'gpw_nn_upsample2_add': (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    'gpw_nn_upsample2_backward': (ctypes.c_int, [ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    'gpw_nn_head': (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp]),
    'gpw_nn_head_backward': (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, _vp, _vp, _vp, _vp, ctypes.c_int, _vp, _vp, ctypes.c_int64, _vp]),
    'gpw_nn_partials': (ctypes.c_int, []),
    'gpw_nn_channel_sum': (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, _vp, _vp, _vp, ctypes.c_int64, _vp]),
    'gpw_nn_pack_input': (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    'gpw_nn_upsample_add_f32': (ctypes.c_int, [ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    'gpw_nn_downsum_f32': (ctypes.c_int, [ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    'gpw_nn_mse': (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int64, _vp]),
    'gpw_nn_unpack_output': (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    'gpw_nn_adam': (ctypes.c_int, [ctypes.c_int64, _vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp, _vp]),
    'gpw_nn_gaussians': (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp, _vp, _vp, _vp]),
}

_lib = None


class GPWError(RuntimeError):
    def __init__(self, code, msg):
        RuntimeError.__init__(self, '%s (code %d)' % (msg, code))
        self.code = code


def load():
    """Load libgpwgrid.so (built in-tree) and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError('libgpwgrid.so is not built (run '
                          '`python -m gpawdft_b200.build`); there is no CPU '
                          'fallback')
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    cache = os.environ.get('GPW_TUNE_CACHE')
    if cache:
        from . import tuning
        tuning._auto(cache)
    return lib


def check(rc):
    if rc != GPW_OK:
        msg = load().gpw_last_error().decode()
        raise GPWError(rc, msg)
