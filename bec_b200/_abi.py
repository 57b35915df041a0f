"""ctypes mirror of include/bec.h (the engine's C ABI).

Every structure here must match include/bec.h field for field; the test suite
checks the sizes against the compiled library.
"""
import ctypes as C

BEC_OK = 0
BEC_ERR_INVALID_ARG = 1
BEC_ERR_UNSUPPORTED_GRID = 2
BEC_ERR_CUDA = 3
BEC_ERR_OUT_OF_MEMORY = 4
BEC_ERR_STATE = 5
BEC_ERR_NUMERICAL = 6
BEC_ERR_NO_DEVICE = 7
BEC_ERR_UNIMPLEMENTED = 8

STATUS_NAMES = {
    0: "BEC_OK", 1: "BEC_ERR_INVALID_ARG", 2: "BEC_ERR_UNSUPPORTED_GRID",
    3: "BEC_ERR_CUDA", 4: "BEC_ERR_OUT_OF_MEMORY", 5: "BEC_ERR_STATE",
    6: "BEC_ERR_NUMERICAL", 7: "BEC_ERR_NO_DEVICE", 8: "BEC_ERR_UNIMPLEMENTED",
}

# host element types of bec_init_groups
BEC_HOST_C128 = 0
BEC_HOST_C64 = 1
BEC_HOST_R32 = 2

BEC_PATH_FP64_PLAIN = 0
BEC_PATH_FP32_BATCHED = 1

BEC_GS_FIXED_STEPS = 0
BEC_GS_MU = 1
BEC_GS_REFERENCE_E = 2
BEC_GS_MU_RESIDUAL = 3
BEC_LR_CONSTANT = 0
BEC_LR_COSINE = 1


class BecParams(C.Structure):
    """ModelParameters (programs/bec_wigner_3d.cuda/defines.h:25-54), SI loss rates."""
    _fields_ = [
        ("a11", C.c_double), ("a12", C.c_double), ("a22", C.c_double),
        ("m", C.c_double),
        ("fx", C.c_double), ("fy", C.c_double), ("fz", C.c_double),
        ("N", C.c_double),
        ("detuning", C.c_double),
        ("gamma111", C.c_double), ("gamma12", C.c_double), ("gamma22", C.c_double),
        ("Va", C.c_double), ("Vb", C.c_double),
        ("nvx", C.c_int32), ("nvy", C.c_int32), ("nvz", C.c_int32),
        ("itmax", C.c_int32),
        ("dt_steady", C.c_double), ("t_equilib", C.c_double), ("dt_evo", C.c_double),
        ("ne", C.c_int32),
        ("loss_noise", C.c_int32),
        ("seed", C.c_uint64),
    ]


class BecDerived(C.Structure):
    """CalculationParameters (defines.h:57-112) in FP64 natural units."""
    _fields_ = [
        ("N", C.c_double),
        ("g11", C.c_double), ("g12", C.c_double), ("g22", C.c_double),
        ("mu", C.c_double),
        ("Va", C.c_double), ("Vb", C.c_double), ("V", C.c_double),
        ("lambda_", C.c_double),
        ("l_rho", C.c_double), ("t_rho", C.c_double),
        ("detuning", C.c_double),
        ("l111", C.c_double), ("l12", C.c_double), ("l22", C.c_double),
        ("xmax", C.c_double), ("ymax", C.c_double), ("zmax", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("dkx", C.c_double), ("dky", C.c_double), ("dkz", C.c_double),
        ("dV", C.c_double),
        ("dt_steady", C.c_double), ("t_equilib", C.c_double), ("dt_evo", C.c_double),
        ("nvx", C.c_int32), ("nvy", C.c_int32), ("nvz", C.c_int32),
        ("cells", C.c_int32),
        ("itmax", C.c_int32),
        ("ne", C.c_int32),
        ("dims", C.c_int32),
        ("n_equil_steps", C.c_int32),
    ]


class BecGsOpts(C.Structure):
    _fields_ = [
        ("mode", C.c_int32), ("max_steps", C.c_int32), ("check_every", C.c_int32),
        ("warm_per_group", C.c_int32),
        ("tol", C.c_double),
        ("warm_start", C.POINTER(C.c_double)),
        ("res_tol", C.c_double),
    ]


class BecGsReport(C.Structure):
    _fields_ = [
        ("steps", C.c_int32), ("converged", C.c_int32),
        ("mu", C.c_double), ("energy", C.c_double), ("N", C.c_double),
        ("residual", C.c_double), ("seconds", C.c_double),
        ("step_residual", C.c_double),
    ]


class BecMoments(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("na", C.c_double), ("nb", C.c_double),
        ("s_re", C.c_double), ("s_im", C.c_double),
    ]


class BecObs(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("N1", C.c_double), ("N2", C.c_double),
        ("Ntotal", C.c_double), ("visibility", C.c_double),
        ("visibility_scan", C.c_double), ("phase", C.c_double),
    ]


class BecSchedule(C.Structure):
    _fields_ = [
        ("n_steps", C.c_int32), ("sample_every", C.c_int32),
        ("pi_pulse_step", C.c_int32), ("axial", C.c_int32),
    ]


def moments_to_array(ms):
    """(n, 5) float array [t, na, nb, s_re, s_im] from a ctypes array of BecMoments."""
    import numpy as np
    return np.array([[m.t, m.na, m.nb, m.s_re, m.s_im] for m in ms], dtype=np.float64)
