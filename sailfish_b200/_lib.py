"""ctypes binding of libsailfish_b200.so (C ABI: include/sailfish_b200.h).

The library is built in tree by ``python -m sailfish_b200.build``.  There is no fallback:
if it is missing or cannot be loaded, importing this module raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsailfish_b200.so")

SF_OK, SF_EINVAL, SF_EDTYPE, SF_ECUDA, SF_ENONFINITE, SF_ETIMEOUT, SF_ENOMEM, SF_EUNSUPPORTED = \
    0, -1, -2, -3, -4, -5, -6, -7
SF_FP64, SF_FP32 = 0, 1

_vp, _d, _i, _i32p = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int32)
_dp = ctypes.POINTER(ctypes.c_double)


class GridDesc(ctypes.Structure):
    _fields_ = [
        ("L", _i), ("M", _i), ("N", _i), ("precision", _i),
        ("h", _dp), ("pm", _dp), ("pn", _dp), ("on_u", _dp), ("om_v", _dp), ("fomn", _dp),
        ("sc_r", _dp), ("sc_w", _dp), ("Cs_r", _dp), ("Cs_w", _dp),
        ("hc", _d), ("Vtransform", _i),
        ("zeta_field_idx2", _i32p), ("uvel_field_type", _i32p), ("vvel_field_type", _i32p),
        ("zeta_copy_idx1", _i32p), ("zeta_copy_idx2", _i32p), ("n_zeta_copy", _i),
        ("ubar_closed_idx", _i32p), ("n_ubar_closed", _i),
        ("vbar_closed_idx", _i32p), ("n_vbar_closed", _i),
        ("ubar_clamped_idx", _i32p), ("n_ubar_clamped", _i),
        ("ubar_grad_idx1", _i32p), ("ubar_grad_idx2", _i32p), ("n_ubar_grad", _i),
        ("vbar_grad_idx1", _i32p), ("n_vbar_grad", _i),
    ]


class GlsParams(ctypes.Structure):
    _fields_ = [(n, _d) for n in ("p", "m", "n", "cmu0", "c1", "c2", "c3m", "c3p", "sigk", "sigp",
                                   "Kmin", "Pmin", "Akv_bak", "Akt_bak", "Akk_bak", "Akp_bak",
                                   "Zos", "Zob", "rdrag2")]


class MlpParams(ctypes.Structure):
    _fields_ = [("W", _vp * 5), ("b", _vp * 5), ("act", ctypes.c_int)]


MLP_ACT = {"gelu": 0, "relu": 1}   # sf_mlp_params.act


class State2D(ctypes.Structure):
    _fields_ = [("zeta", _vp * 3), ("ubar", _vp * 3), ("vbar", _vp * 3), ("rzeta", _vp * 3),
                ("rubar", _vp * 3), ("rvbar", _vp * 3),
                ("Zt_avg1", _vp), ("DU_avg1", _vp), ("DV_avg1", _vp)]


# name -> argtypes (after the context pointer for the kernel entry points)
SIGNATURES = {
    "sf_ctx_create": [ctypes.POINTER(GridDesc), ctypes.POINTER(_vp)],
    "sf_ctx_destroy": [_vp],
    "sf_last_error": [],
    "sf_version": [],
    "sf_ctx_precision": [_vp],
    "sf_zeta_rhs": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _d, _vp, _vp],
    "sf_zeta_pred": [_vp, _d, _vp, _vp, _vp, _vp],
    "sf_momentum_rhs": [_vp, _vp, _vp, _vp, _vp, _d, _d, _vp],
    "sf_momentum_pred": [_vp, _d, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "sf_am3": [_vp, _d, _vp, _vp, _vp, _vp, _vp],
    "sf_zetabc": [_vp, _vp, _vp],
    "sf_barotropic_velocity_bc": [_vp, _vp, _vp, _d, _vp],
    "sf_step2d_predictor": [_vp, ctypes.POINTER(State2D), _d, _d, _i, _vp],
    "sf_step2d_corrector": [_vp, ctypes.POINTER(State2D), _d, _d, _d, _vp],
    "sf_barotropic_substep": [_vp, ctypes.POINTER(State2D), _d, _d, _d, _i, _vp],
    "sf_barotropic_loop": [_vp, ctypes.POINTER(State2D), _i, _dp, _d, _dp, _vp],
    "sf_roms_barotropic_loop": [_vp, ctypes.POINTER(State2D), _vp, _vp, _vp, _vp, _d, _i, _dp,
                                _dp, _d, _vp],
    "sf_roms_step2d": [_vp, ctypes.POINTER(State2D), _vp, _vp, _d, _d, _i, _vp],
    "sf_roms_stress3d": [_vp] * 7 + [_d, _vp],
    "sf_roms_rhs3d": [_vp] * 9,
    "sf_roms_step3d_uv": [_vp] * 19 + [_i, _i, _d, _d, _vp],
    "sf_roms_closed_walls": [_vp] * 4,
    "sf_rhs3d": [_vp] * 10,
    "sf_set_maxflux": [_vp] * 7,
    "sf_omega": [_vp] * 6,
    "sf_maxflux_omega": [_vp] * 12,
    "sf_set_zeta": [_vp] * 5,
    "sf_set_depth": [_vp] * 6,
    "sf_check_state": [_vp] * 6 + [_d, _d, _vp],
    "sf_step3d_uv": [_vp] * 16 + [_i, _i, _d, _d, _vp],
    "sf_lateral_uv_bc": [_vp, _d, _vp, _vp, _vp],
    "sf_step3d_uv_bc": [_vp] * 14 + [_i, _i, _d, _d, _d, _vp],
    "sf_gls_corrector": [_vp, ctypes.POINTER(GlsParams), _d] + [_vp] * 14 + [_vp],
    "sf_gls_corrector_cols": [_vp, ctypes.POINTER(GlsParams), _d] + [_vp] * 15 + [_vp],
    "sf_gls_corrector_list": [_vp, ctypes.POINTER(GlsParams), _d] + [_vp] * 16 + [_vp],
    "sf_analytic_bvf": [_vp, _vp, _d, _d, _d, _d, _vp, _vp],
    "sf_gls_predictor": [_vp, _d, _i] + [_vp] * 13 + [_vp],
    "sf_gls_advect": [_vp, ctypes.POINTER(GlsParams), _d, _d] + [_vp] * 7 + [_vp],
    "sf_gls_corrector_nnew": [_vp, ctypes.POINTER(GlsParams), _d] + [_vp] * 16 + [_vp],
    "sf_obc_volcons": [_vp, _vp, _vp, _vp, _i, _i, _vp, _vp],
    "sf_ctx_set_graphs": [_vp, _i],
    "sf_ctx_set_pdl": [_vp, _i],
    "sf_ctx_set_fused": [_vp, _i],
    "sf_ctx_set_bulk": [_vp, _i],
    "sf_ctx_tune": [_vp, _i, _i],
    "sf_ctx_fused_available": [_vp],
    "sf_ctx_create_ensemble": [ctypes.POINTER(GridDesc), _i, ctypes.POINTER(_vp)],
    "sf_ctx_members": [_vp],
    "sf_ctx_set_tile": [_vp, _i],
    "sf_ctx_member_layout": [_vp, _vp, _vp, _vp, _vp],
    "sf_mlp_last_error": [],
    "sf_mlp_gemm": [_i, _i, _vp, _i, ctypes.c_long, ctypes.c_long, _vp, _i, ctypes.c_long,
                    ctypes.c_long, _vp, _i, _vp, ctypes.c_long, _vp, ctypes.c_long, _vp, _vp],
    "sf_mlp_forward": [ctypes.POINTER(MlpParams), _i, _vp, _vp, _vp, _vp, _vp, _vp],
    "sf_mlp_infer": [ctypes.POINTER(MlpParams), _i, _vp, _vp, _vp, _vp],
    "sf_mlp_backward": [ctypes.POINTER(MlpParams), _i, _vp, _vp, _vp, _vp, ctypes.POINTER(_vp),
                        ctypes.POINTER(_vp), _vp, _vp, _vp],
    "sf_mlp_backward_static": [ctypes.POINTER(MlpParams), _i, _vp, _vp, _vp, _vp,
                               ctypes.POINTER(_vp), ctypes.POINTER(_vp), _vp, _vp],
    "sf_mlp_mse": [_i, _i, _vp, _vp, _vp, _vp, _vp],
    "sf_mlp_adam": [ctypes.c_long, _vp, _vp, _vp, _vp, _vp, ctypes.c_float, ctypes.c_float,
                    ctypes.c_float, _i, ctypes.c_float, _vp],
    "sf_closure_features": [_vp] * 9,
    "sf_closure_apply": [_vp] * 6,
    "sf_closure_range_mask": [_vp, _vp, _i, _vp, _vp, _vp, _vp],
    "sf_closure_step": [_vp, ctypes.POINTER(MlpParams)] + [_vp] * 6 + [_i] + [_vp] * 9,
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("libsailfish_b200.so is not built (run: python -m sailfish_b200.build)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = ctypes.c_char_p if name.endswith("last_error") else ctypes.c_int
    return lib


lib = _load()


class SailfishError(RuntimeError):
    """A failed library call (status code and the library's error text), or a caller error
    found on the host (message only, status SF_EINVAL)."""

    def __init__(self, code, where=None):
        if where is None:
            super().__init__(str(code))
            self.code = SF_EINVAL
            return
        msg = lib.sf_last_error().decode(errors="replace")
        super().__init__("%s failed (status %d): %s" % (where, code, msg))
        self.code = code


def check(code, where):
    if code != SF_OK:
        raise SailfishError(code, where)
    return code
