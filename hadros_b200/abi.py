"""ctypes mirror of include/hadros_b200.h (structures and constants only).

Importing this module loads nothing; hadros_b200.lib() loads the library.
"""
from __future__ import annotations

import ctypes as C

ABI_VERSION = 2

OK, E_ARG, E_IO, E_CUDA, E_RANGE, E_TIMEOUT, E_NOMEM, E_STATE = range(8)

PROFILES = ("gaussian", "powerlaw", "gaussian_funnel", "powerlaw_funnel",
            "gaussian_envelope", "powerlaw_envelope", "powerlaw_funnel_envelope",
            "collapsar_ndaf_like")
SOURCES = ("inner_ring", "funnel_wall", "jet_base", "shock_layer", "density_weighted")
SPECTRA = ("monochromatic", "powerlaw", "powerlaw_cutoff")

PRECISION_FP64 = 0
PRECISION_MIXED = 1

FATE_ESCAPED, FATE_CAPTURED, FATE_TRUNCATED = 0, 1, 2

TRANSFER_AUTO, TRANSFER_IN_LOOP, TRANSFER_DEFERRED = 0, 1, 2


class HadrosParams(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("max_steps", C.c_int32),
        ("profile_kind", C.c_int32),
        ("source_kind", C.c_int32),
        ("spectral_kind", C.c_int32),
        ("n_bins", C.c_int32),
        ("precision", C.c_int32),
        ("fast_geodesic", C.c_int32),
        ("a_spin", C.c_double),
        ("r_obs_rg", C.c_double),
        ("theta_obs_rad", C.c_double),
        ("fov_deg", C.c_double),
        ("r_max_rg", C.c_double),
        ("h", C.c_double),
        ("tolerance", C.c_double),
        ("Enu_obs_GeV", C.c_double),
        ("M_bh_msun", C.c_double),
        ("rho0_gcm3", C.c_double),
        ("r0_rg", C.c_double),
        ("sigma_r_rg", C.c_double),
        ("H_over_R", C.c_double),
        ("radial_power", C.c_double),
        ("funnel_depletion", C.c_double),
        ("funnel_theta_rad", C.c_double),
        ("envelope_rho0_gcm3", C.c_double),
        ("envelope_alpha", C.c_double),
        ("torus_r_min_rg", C.c_double),
        ("torus_r_max_rg", C.c_double),
        ("rho_floor_gcm3", C.c_double),
        ("src_r_center_rg", C.c_double),
        ("src_sigma_r_rg", C.c_double),
        ("src_theta_width_rad", C.c_double),
        ("src_powerlaw", C.c_double),
        ("src_emax_GeV", C.c_double),
        ("src_norm", C.c_double),
        ("src_funnel_theta_rad", C.c_double),
        ("src_density_power_q", C.c_double),
        ("src_radial_power_s", C.c_double),
        ("src_rho_ref_gcm3", C.c_double),
        ("src_cutoff_min", C.c_double),
        ("src_cutoff_max", C.c_double),
        ("src_gradient_dr_rg", C.c_double),
        ("src_gradient_dtheta_rad", C.c_double),
        ("spec_gamma", C.c_double),
        ("spec_ecut_GeV", C.c_double),
        ("spec_e_min_GeV", C.c_double),
        ("spec_e_max_GeV", C.c_double),
        ("mev_channel", C.c_int32),
        ("mev_model", C.c_int32),
        ("mev_flavor", C.c_int32),
        ("mev_thermal_profile", C.c_int32),
        ("mev_ye_profile", C.c_int32),
        ("mev_spectral_mode", C.c_int32),
        ("mev_n_bins", C.c_int32),
        ("mev_flags", C.c_uint32),
        ("mev_Enu_obs_MeV", C.c_double),
        ("mev_norm", C.c_double),
        ("mev_sigma_abs0_cm2", C.c_double),
        ("mev_sigma_scat0_cm2", C.c_double),
        ("mev_neutrinosphere_tau", C.c_double),
        ("mev_T0_MeV", C.c_double),
        ("mev_T_floor_MeV", C.c_double),
        ("mev_T_power", C.c_double),
        ("mev_Ye_torus", C.c_double),
        ("mev_Ye_funnel", C.c_double),
        ("mev_Ye_envelope", C.c_double),
        ("mev_Ye_floor", C.c_double),
        ("mev_Ye_ceil", C.c_double),
        ("mev_E_min_MeV", C.c_double),
        ("mev_E_max_MeV", C.c_double),
    ]

    def copy(self) -> "HadrosParams":
        q = HadrosParams()
        C.memmove(C.byref(q), C.byref(self), C.sizeof(HadrosParams))
        return q

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class HadrosImageOut(C.Structure):
    _fields_ = [
        ("tau", C.c_void_p),
        ("P_surv", C.c_void_p),
        ("I_obs", C.c_void_p),
        ("fate", C.c_void_p),
        ("steps", C.c_void_p),
        ("attempts", C.c_void_p),
        ("tau_E", C.c_void_p),
        ("I_E", C.c_void_p),
        ("tau_mev", C.c_void_p),
        ("P_surv_mev", C.c_void_p),
        ("I_obs_mev", C.c_void_p),
        ("r_nu", C.c_void_p),
        ("leakage", C.c_void_p),
    ]


# MeV thermal channel (enum hadros_mev_* of include/hadros_b200.h)
MEV_TOY, MEV_PHYSICAL = 0, 1
MEV_NU_E, MEV_ANTI_NU_E, MEV_NU_X = 0, 1, 2
MEV_MONOCHROMATIC, MEV_FERMI_DIRAC_BAND = 0, 1
MEV_FLAG_BITS = {"urca": 1 << 0, "pair": 1 << 1, "brems": 1 << 2, "absorption": 1 << 3, "scattering": 1 << 4,
                 "degeneracy_correction": 1 << 5, "abs_n": 1 << 6, "abs_p": 1 << 7, "scat_n": 1 << 8,
                 "scat_p": 1 << 9, "scat_e": 1 << 10}
MEV_FLAGS_DEFAULT = 0x7DF
MEV_OUTPUTS = ("tau_mev", "P_surv_mev", "I_obs_mev", "r_nu", "leakage")


ORDER_ROWS, ORDER_TILES, ORDER_COST = 0, 1, 2


class HadrosSchedule(C.Structure):
    _fields_ = [("blocks_per_sm", C.c_int32), ("order", C.c_int32), ("coarse_stride", C.c_int32),
                ("camera_order", C.c_int32)]


class HadrosStats(C.Structure):
    _fields_ = [
        ("kernel_ms", C.c_double),
        ("total_ms", C.c_double),
        ("rays", C.c_int64),
        ("accepted_steps", C.c_int64),
        ("attempts", C.c_int64),
        ("h2d_bytes", C.c_int64),
        ("d2h_bytes", C.c_int64),
        ("launches", C.c_int32),
        ("aborted_rays", C.c_int32),
    ]


# Every function the header declares: name -> (restype, argtypes).
P = C.POINTER
class HadrosMlpNorm(C.Structure):
    _fields_ = [("feat_mu", C.c_float * 16), ("feat_inv_sd", C.c_float * 16),
                ("out_mu", C.c_float * 2), ("out_sd", C.c_float * 2), ("out_floor", C.c_float * 2)]


class HadrosAdam(C.Structure):
    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float)]


class HadrosTrainSched(C.Structure):
    _fields_ = [("lr_max", C.c_float), ("lr_min", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float),
                ("eps", C.c_float), ("total_steps", C.c_int64), ("steps_per_epoch", C.c_int64)]


class HadrosSurrogateOut(C.Structure):
    _fields_ = [("ln_tau_E", C.c_void_p), ("ln_I_E", C.c_void_p), ("tau", C.c_void_p),
                ("P_surv", C.c_void_p), ("I_obs", C.c_void_p), ("spread", C.c_void_p),
                ("fallback_ids", C.c_void_p), ("counters", C.c_void_p)]


SIGNATURES = {
    "hadros_abi_version": (C.c_int32, []),
    "hadros_status_string": (C.c_char_p, [C.c_int32]),
    "hadros_last_error": (C.c_char_p, []),
    "hadros_params_default": (None, [P(HadrosParams)]),
    "hadros_params_validate": (C.c_int32, [P(HadrosParams)]),
    "hadros_parse_profile": (C.c_int32, [C.c_char_p, P(C.c_int32)]),
    "hadros_parse_source": (C.c_int32, [C.c_char_p, P(C.c_int32)]),
    "hadros_parse_spectral": (C.c_int32, [C.c_char_p, P(C.c_int32)]),
    "hadros_profile_name": (C.c_char_p, [C.c_int32]),
    "hadros_source_name": (C.c_char_p, [C.c_int32]),
    "hadros_spectral_name": (C.c_char_p, [C.c_int32]),
    "hadros_parse_mev_model": (C.c_int32, [C.c_char_p, P(C.c_int32)]),
    "hadros_parse_mev_flavor": (C.c_int32, [C.c_char_p, P(C.c_int32)]),
    "hadros_parse_mev_thermal": (C.c_int32, [C.c_char_p, P(C.c_int32)]),
    "hadros_parse_mev_ye": (C.c_int32, [C.c_char_p, P(C.c_int32)]),
    "hadros_parse_mev_spectral": (C.c_int32, [C.c_char_p, P(C.c_int32)]),
    "hadros_mev_model_name": (C.c_char_p, [C.c_int32]),
    "hadros_mev_flavor_name": (C.c_char_p, [C.c_int32]),
    "hadros_mev_thermal_name": (C.c_char_p, [C.c_int32]),
    "hadros_mev_ye_name": (C.c_char_p, [C.c_int32]),
    "hadros_mev_spectral_name": (C.c_char_p, [C.c_int32]),
    "hadros_sigma_load": (C.c_int32, [C.c_char_p, P(C.c_void_p)]),
    "hadros_sigma_from_arrays": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                             P(C.c_void_p)]),
    "hadros_sigma_info": (C.c_int32, [C.c_void_p, P(C.c_int32), P(C.c_double), P(C.c_double)]),
    "hadros_sigma_eval_cm2": (C.c_int32, [C.c_void_p, C.c_double, P(C.c_double)]),
    "hadros_sigma_destroy": (None, [C.c_void_p]),
    "hadros_spectral_bins": (C.c_int32, [P(HadrosParams), C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p, P(C.c_int32)]),
    "hadros_ctx_create": (C.c_int32, [C.c_int32, P(C.c_void_p)]),
    "hadros_ctx_destroy": (None, [C.c_void_p]),
    "hadros_ctx_stats": (C.c_int32, [C.c_void_p, P(HadrosStats)]),
    "hadros_ctx_set_transfer": (C.c_int32, [C.c_void_p, C.c_int32]),
    "hadros_ctx_set_attempt_budget": (C.c_int32, [C.c_void_p, C.c_int64]),
    "hadros_image": (C.c_int32, [C.c_void_p, P(HadrosParams), C.c_void_p, P(HadrosImageOut)]),
    "hadros_image_pixels": (C.c_int32, [C.c_void_p, P(HadrosParams), C.c_void_p, C.c_void_p,
                                        C.c_int32, P(HadrosImageOut)]),
    "hadros_image_device": (C.c_int32, [C.c_void_p, P(HadrosParams), C.c_void_p,
                                        P(HadrosImageOut), C.c_void_p]),
    "hadros_image_pixels_device": (C.c_int32, [C.c_void_p, P(HadrosParams), C.c_void_p, C.c_void_p,
                                               C.c_int32, P(HadrosImageOut), C.c_void_p]),
    "hadros_ctx_synchronize": (C.c_int32, [C.c_void_p]),
    "hadros_batch": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, P(HadrosImageOut)]),
    "hadros_batch_device": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                        P(HadrosImageOut), C.c_void_p]),
    "hadros_batch_pixels": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                        C.c_void_p, P(HadrosImageOut)]),
    "hadros_image_device_noalloc": (C.c_int32, [P(HadrosParams), C.c_void_p, P(HadrosImageOut),
                                                C.c_void_p]),
    "hadros_schedule_default": (None, [P(HadrosSchedule)]),
    "hadros_plan_create": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                       P(HadrosSchedule), P(C.c_void_p)]),
    "hadros_plan_info": (C.c_int32, [C.c_void_p, P(C.c_int64), P(C.c_int64), P(C.c_int32),
                                     P(C.c_int32)]),
    "hadros_plan_launch": (C.c_int32, [C.c_void_p, P(HadrosImageOut), C.c_void_p]),
    "hadros_plan_counters": (C.c_int32, [C.c_void_p, C.c_void_p, P(C.c_int64), P(C.c_int64),
                                         P(C.c_int32)]),
    "hadros_plan_destroy": (None, [C.c_void_p]),
    "hadros_trace_paths": (C.c_int32, [C.c_void_p, P(HadrosParams), C.c_void_p, C.c_int32, C.c_int32,
                                       C.c_void_p, C.c_void_p, C.c_void_p]),
    "hadros_transfer_paths": (C.c_int32, [C.c_void_p, P(HadrosParams), C.c_void_p, C.c_int32,
                                          C.c_void_p, C.c_void_p, C.c_void_p, P(HadrosImageOut)]),
    "hadros_write_kgeo": (C.c_int32, [C.c_char_p, P(HadrosParams), C.c_int32, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]),
    "hadros_write_kgeo_rays": (C.c_int32, [C.c_char_p, P(HadrosParams), C.c_int32, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_int32]),
    "hadros_kgeo_info": (C.c_int32, [C.c_char_p, P(C.c_int32), P(C.c_int32), P(C.c_double),
                                     P(C.c_int32), P(C.c_int64)]),
    "hadros_read_kgeo": (C.c_int32, [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]),
    "hadros_image_filename": (C.c_int32, [P(HadrosParams), C.c_int32, C.c_char_p, C.c_double,
                                          C.c_double, C.c_char_p, C.c_char_p, C.c_int32]),
    "hadros_write_dat": (C.c_int32, [C.c_char_p, P(HadrosParams), C.c_char_p, C.c_double,
                                     C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hadros_write_kimg": (C.c_int32, [C.c_char_p, P(HadrosParams), C.c_double, C.c_double,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hadros_write_dat_mev": (C.c_int32, [C.c_char_p, P(HadrosParams), C.c_char_p, P(HadrosImageOut)]),
    "hadros_write_kimg_mev": (C.c_int32, [C.c_char_p, P(HadrosParams), P(HadrosImageOut)]),
    "hadros_mlp_param_count": (C.c_int64, []),
    "hadros_mlp_packed_count": (C.c_int64, []),
    "hadros_mlp_workspace_bytes": (C.c_int64, [C.c_int64]),
    "hadros_mlp_layout": (C.c_int32, [C.c_void_p, C.c_int32]),
    "hadros_mlp_pack": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "hadros_mlp_featurize": (C.c_int32, [C.c_void_p, C.c_int64, P(HadrosMlpNorm), C.c_void_p,
                                         C.c_void_p]),
    "hadros_mlp_raw_features": (C.c_int32, [P(HadrosParams), C.c_void_p, C.c_void_p, C.c_int64,
                                            C.c_void_p, C.c_void_p]),
    "hadros_mlp_forward": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                       C.c_void_p, C.c_void_p]),
    "hadros_mlp_backward": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p]),
    "hadros_mlp_loss": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                    C.c_void_p, C.c_void_p]),
    "hadros_mlp_adam": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, P(HadrosAdam),
                                    C.c_int64, C.c_void_p]),
    "hadros_mlp_train_step": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_int64, P(HadrosAdam), C.c_int64,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p]),
    "hadros_mlp_members_workspace_bytes": (C.c_int64, [C.c_int32, C.c_int64]),
    "hadros_mlp_train_members": (C.c_int32, [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, P(HadrosAdam), C.c_int64, C.c_void_p,
                                             C.c_void_p, C.c_void_p]),
    "hadros_mlp_train_members_dev": (C.c_int32, [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_void_p, P(HadrosTrainSched), C.c_void_p,
                                                 C.c_void_p, C.c_void_p, C.c_void_p]),
    "hadros_mlp_image_bytes": (C.c_int64, []),
    "hadros_surrogate_schedule": (C.c_int32, [C.c_int32]),
    "hadros_mlp_pack_image": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "hadros_surrogate_image": (C.c_int32, [P(HadrosParams), C.c_void_p, C.c_int32, C.c_void_p,
                                           C.c_void_p, P(HadrosMlpNorm), C.c_int64, C.c_int64,
                                           C.c_float, C.c_int32, P(HadrosSurrogateOut), C.c_void_p]),
}
