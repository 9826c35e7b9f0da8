"""ctypes binding of the C ABI in include/pgfem_gpu.h.

This is harness plumbing for tests and benchmarks: every numerical operation
runs inside libpgfem_gpu.so (setup on the host in C++, assembly on the GPU).
Loading fails loudly when the library is missing; there is no fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpgfem_gpu.so")

MODEL_HE, MODEL_J2, MODEL_CP = 0, 1, 2
SCATTER_ATOMIC, SCATTER_COLOUR = 0, 1

ERRORS = {-1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "EPATTERN", -5: "ENODEV", -6: "ELIMIT", -7: "ETIMEOUT",
          -8: "EFORMAT"}


class PgfemError(RuntimeError):
    def __init__(self, fn, code):
        super().__init__("%s failed: %s (%d)" % (fn, ERRORS.get(code, "?"), code))
        self.code = code


class MaterialDesc(C.Structure):
    _fields_ = [("model", C.c_int), ("E", C.c_double), ("nu", C.c_double),
                ("sigma_y", C.c_double), ("H", C.c_double),
                ("gamma_dot_0", C.c_double), ("m", C.c_double), ("G0", C.c_double),
                ("g0", C.c_double), ("gs_0", C.c_double), ("gamma_dot_s", C.c_double),
                ("w", C.c_double), ("cp_tol", C.c_double), ("cp_max_iter", C.c_int),
                ("dev_pot", C.c_int), ("vol_pot", C.c_int)]


class MeshDesc(C.Structure):
    _fields_ = [("nn", C.c_long), ("ne", C.c_long), ("nne", C.c_int),
                ("X", C.POINTER(C.c_double)), ("conn", C.POINTER(C.c_int)),
                ("dof_id", C.POINTER(C.c_long)), ("ndof", C.c_long), ("npres", C.c_long),
                ("F0", C.POINTER(C.c_double)), ("R_cp", C.POINTER(C.c_double))]


class Status(C.Structure):
    _fields_ = [("inverted", C.c_long), ("nonconverged", C.c_long),
                ("bad_diagonal", C.c_long), ("other", C.c_long)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}

    def ok(self):
        return self.inverted == 0 and self.nonconverged == 0 and self.bad_diagonal == 0 and self.other == 0


_lib = None

_P = C.c_void_p


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError("libpgfem_gpu.so not built: run pgfem-3d_b200/build.py")
        L = C.CDLL(LIB_PATH)
        sig = {
            "pgfem_gpu_state_size": (C.c_int, [C.c_int]),
            "pgfem_generate_dof_ids": (C.c_long, [C.c_long, C.c_long, C.c_int, _P, _P, _P]),
            "pgfem_psparse_apai": (C.c_long, [C.c_long, C.c_int, _P, _P, C.c_long, _P, _P]),
            "pgfem_mesh_box_tet": (C.c_int, [C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P]),
            "pgfem_gpu_create": (C.c_int, [_P, _P, _P, _P, C.c_long, _P]),
            "pgfem_gpu_destroy": (C.c_int, [_P]),
            "pgfem_gpu_set_scatter_mode": (C.c_int, [_P, C.c_int]),
            "pgfem_gpu_set_wait_test": (C.c_int, [_P, C.c_double, C.c_int]),
            "pgfem_gpu_set_neumann": (C.c_int, [_P, C.c_long, _P, _P, _P, C.c_int, _P, _P]),
            "pgfem_cp_resolved_shear": (C.c_int, [_P, C.c_long, _P, _P, _P, _P, _P, _P]),
            "pgfem_gpu_assemble_RK_transient": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, C.c_double, C.c_double,
                                                          C.c_double, C.c_double, _P, _P, _P]),
            "pgfem_gpu_set_neumann_loads": (C.c_int, [_P, C.c_int, _P]),
            "pgfem_gpu_set_neumann_load_history": (C.c_int, [_P, C.c_int, _P, _P]),
            "pgfem_gpu_set_three_field": (C.c_int, [_P, _P, _P]),
            "pgfem_gpu_get_three_field": (C.c_int, [_P, _P, _P]),
            "pgfem_gpu_three_field_enabled": (C.c_int, [_P]),
            "pgfem_gpu_three_field_increments": (C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
            "pgfem_gpu_three_field_update_device": (C.c_int, [_P, _P, _P, _P, _P, _P]),
            "pgfem_gpu_set_three_field_history": (C.c_int, [_P, _P, _P, _P, _P]),
            "pgfem_gpu_assemble_RK_transient_device": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, C.c_double, C.c_double,
                                                                 C.c_double, C.c_double, _P, _P, _P]),
            "pgfem_gpu_three_field_increments_transient": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, C.c_double,
                                                                     C.c_double, C.c_double, _P, _P, _P]),
            "pgfem_mlp_set_wait_test": (C.c_int, [_P, C.c_double, C.c_int]),
            "pgfem_gpu_device_bytes": (C.c_long, [_P]),
            "pgfem_gpu_nnz": (C.c_long, [_P]),
            "pgfem_gpu_set_state": (C.c_int, [_P, _P]),
            "pgfem_gpu_get_state": (C.c_int, [_P, C.c_int, _P]),
            "pgfem_gpu_set_state_nm1": (C.c_int, [_P, _P]),
            "pgfem_gpu_commit_state": (C.c_int, [_P]),
            "pgfem_gpu_reset_state": (C.c_int, [_P]),
            "pgfem_gpu_assemble_R": (C.c_int, [_P, _P, _P, C.c_double, _P, _P]),
            "pgfem_gpu_assemble_RK": (C.c_int, [_P, _P, _P, C.c_double, _P, _P, _P]),
            "pgfem_gpu_assemble_RK_device": (C.c_int, [_P, _P, _P, C.c_double, _P, _P, _P]),
            "pgfem_gpu_read_status": (C.c_int, [_P, _P, C.c_int]),
            "pgfem_gpu_launches_per_assembly": (C.c_int, [_P]),
            "pgfem_gpu_stiffmatel_fd": (C.c_int, [_P, C.c_long, _P, _P, _P, C.c_double, _P, _P, _P]),
            "pgfem_gpu_resid_on_elem": (C.c_int, [_P, C.c_long, _P, _P, _P, C.c_double, _P, _P]),
            "pgfem_gpu_cm_integrate": (C.c_int, [_P, C.c_long, _P, C.c_double, _P, _P, _P, _P, _P, _P]),
            "pgfem_gpu_set_timing": (C.c_int, [_P, C.c_int]),
            "pgfem_gpu_kernel_time": (C.c_int, [_P, _P, _P, C.c_int]),
            "pgfem_gpu_fp64_peak": (C.c_int, [_P]),
            "pgfem_gpu_binary_version": (C.c_int, [_P]),
            "pgfem_gpu_set_cp_guess": (C.c_int, [_P, _P]),
            "pgfem_gpu_get_cp_iterations": (C.c_int, [_P, _P, _P]),
            "pgfem_gpu_cp_integrate_noalloc": (C.c_int, [_P, C.c_long, _P, _P, _P, C.c_double, _P, _P, _P, _P,
                                                         _P]),
            "pgfem_mlp_num_params": (C.c_long, []),
            "pgfem_mlp_create": (C.c_int, [C.c_ulonglong, _P]),
            "pgfem_mlp_destroy": (C.c_int, [_P]),
            "pgfem_mlp_set_params": (C.c_int, [_P, _P]),
            "pgfem_mlp_get_params": (C.c_int, [_P, _P]),
            "pgfem_mlp_set_scaling": (C.c_int, [_P, _P, _P, _P]),
            "pgfem_mlp_get_scaling": (C.c_int, [_P, _P, _P, _P]),
            "pgfem_mlp_fit_scaling": (C.c_int, [_P, C.c_long, _P, _P]),
            "pgfem_mlp_predict_device": (C.c_int, [_P, C.c_long, _P, _P, _P]),
            "pgfem_mlp_predict": (C.c_int, [_P, C.c_long, _P, _P]),
            "pgfem_mlp_loss_grad": (C.c_int, [_P, C.c_long, _P, _P, _P, _P]),
            "pgfem_mlp_train_device": (C.c_int, [_P, C.c_long, _P, _P, _P, _P]),
            "pgfem_gpu_set_cp_warm_limit": (C.c_int, [_P, C.c_int]),
            "pgfem_gpu_set_cp_surrogate": (C.c_int, [_P, _P]),
            "pgfem_gpu_cp_training_pairs": (C.c_int, [_P, _P, _P]),
            "pgfem_gpu_get_cp_fallbacks": (C.c_int, [_P, _P]),
            "pgfem_gpu_set_mesh_groups": (C.c_int, [_P, C.c_int, _P, _P]),
            "pgfem_gpu_set_schedule": (C.c_int, [_P, C.c_int, C.c_int]),
            "pgfem_gpu_get_schedule": (C.c_int, [_P, _P, _P]),
            "pgfem_gpu_graph_create": (C.c_int, [_P, _P, _P, C.c_double, _P, _P, _P]),
            "pgfem_gpu_graph_launch": (C.c_int, [_P, _P]),
            "pgfem_gpu_graph_destroy": (C.c_int, [_P]),
            "pgfem_gpu_autotune": (C.c_int, [_P, _P, _P, C.c_double, _P, _P, C.c_int, _P, _P, _P]),
            "pgfem_gpu_solver_create": (C.c_int, [_P, _P, C.c_long, _P, _P]),
            "pgfem_gpu_solver_destroy": (C.c_int, [_P]),
            "pgfem_gpu_solver_device_bytes": (C.c_long, [_P]),
            "pgfem_gpu_spmv": (C.c_int, [_P, _P, _P, _P, _P]),
            "pgfem_gpu_solve": (C.c_int, [_P, _P, _P, _P, _P, _P]),
            "pgfem_gpu_newton_step": (C.c_int, [_P, _P, _P, _P, C.c_double, _P, _P, _P]),
            "pgfem_input_last_error": (C.c_char_p, []),
            "pgfem_input_read_mesh": (C.c_int, [C.c_char_p, C.c_int, _P]),
            "pgfem_input_read_mesh_bc": (C.c_int, [C.c_char_p, C.c_int, C.c_char_p, _P]),
            "pgfem_input_read_mesh_mp": (C.c_int, [C.c_char_p, C.c_int, C.c_char_p, C.c_int, _P, C.c_int, _P]),
            "pgfem_input_read_multiphysics": (C.c_int, [C.c_char_p, C.c_int, _P, _P, _P]),
            "pgfem_input_get_info": (C.c_int, [_P, _P]),
            "pgfem_input_get_mesh": (C.c_int, [_P, _P, _P, _P, _P]),
            "pgfem_input_get_elements": (C.c_int, [_P, _P, _P, _P, _P]),
            "pgfem_input_get_materials": (C.c_int, [_P, _P, _P, _P]),
            "pgfem_input_read_orientations": (C.c_int, [_P, C.c_char_p, _P, _P]),
            "pgfem_input_destroy": (None, [_P]),
            "pgfem_input_get_partition": (C.c_int, [_P, C.c_int, _P, _P, _P]),
            "pgfem_input_get_periodic": (C.c_int, [_P, _P]),
            "pgfem_input_get_element_faces": (C.c_int, [_P, _P, _P]),
            "pgfem_input_read_nbc": (C.c_int, [C.c_char_p, C.c_char_p, _P]),
            "pgfem_nbc_get_features": (C.c_int, [_P, _P, _P, _P, _P]),
            "pgfem_nbc_faces": (C.c_int, [_P, _P, _P, _P, _P, _P]),
            "pgfem_nbc_load_values": (C.c_int, [_P, C.c_double, _P]),
            "pgfem_nbc_destroy": (None, [_P]),
            "pgfem_load_expression": (C.c_int, [C.c_char_p, C.c_double, _P]),
            "pgfem_euler_rotation": (C.c_int, [C.c_long, _P, _P]),
            "pgfem_input_read_solver_file": (C.c_int, [C.c_char_p, C.c_long, _P, _P, _P, _P, _P]),
            "pgfem_input_j2_material": (C.c_int, [_P, C.c_double, C.c_double, C.c_int, _P]),
            "pgfem_input_read_model_params": (C.c_int, [C.c_char_p, C.c_int, _P, _P]),
            "pgfem_restart_block_size": (C.c_int, [C.c_int]),
            "pgfem_restart_format": (C.c_int, [C.c_char_p, C.c_long, C.c_long, C.c_int, C.c_int, _P, _P, _P]),
            "pgfem_restart_parse": (C.c_int, [C.c_char_p, C.c_long, C.c_long, C.c_int, C.c_int, _P, _P, _P]),
            "pgfem_gpu_write_restart": (C.c_int, [_P, C.c_char_p, _P, _P, _P, _P, _P]),
            "pgfem_restart_write_partitions": (C.c_int, [_P, C.c_char_p, C.c_int, C.c_int, C.c_int, _P, _P, _P]),
            "pgfem_gpu_read_restart": (C.c_int, [_P, C.c_char_p, _P, _P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    return a  # integer device pointer


def _check(fn, r):
    if r < 0:
        raise PgfemError(fn, r)
    return r


def material(model, E=200e3, nu=0.3, sigma_y=0.0, H=0.0, gamma_dot_0=0.0, m=1.0, G0=0.0, g0=0.0,
             gs_0=0.0, gamma_dot_s=1.0, w=0.0, cp_tol=1e-10, cp_max_iter=25, dev_pot=1, vol_pot=99):
    """Material record; dev_pot is the reference's devPotFlag for HE (1
    neo-Hookean, 2 linear deviatoric potential), vol_pot its volPotFlag for HE
    and J2 (99 U_Common, 2 and 3 the Doll-Schweizerhof forms)."""
    return MaterialDesc(model, E, nu, sigma_y, H, gamma_dot_0, m, G0, g0, gs_0, gamma_dot_s, w,
                        cp_tol, cp_max_iter, dev_pot, vol_pot)


# ---------------------------------------------------------------- setup ----
def mesh_box_tet(n, nne, periodic=False):
    """Structured unit-cube mesh (6 tets per cell).  Returns X (nn,3), conn (ne,nne), Pr (nn,)."""
    nn = C.c_long()
    ne = C.c_long()
    _check("pgfem_mesh_box_tet", lib().pgfem_mesh_box_tet(n, nne, int(periodic), C.byref(nn), C.byref(ne),
                                                          None, None, None))
    X = np.zeros((nn.value, 3))
    conn = np.zeros((ne.value, nne), dtype=np.int32)
    Pr = np.zeros(nn.value, dtype=np.int64)
    _check("pgfem_mesh_box_tet", lib().pgfem_mesh_box_tet(n, nne, int(periodic), C.byref(nn), C.byref(ne),
                                                          _ptr(X), _ptr(conn), _ptr(Pr)))
    return X, conn, Pr


def generate_dof_ids(conn, nn, codes, Pr=None):
    """codes (nn,3) int64: 0 free, 1 fixed, <0 prescribed.  Returns (ids, ndof)."""
    ids = np.ascontiguousarray(codes, dtype=np.int64).copy()
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    Pr = None if Pr is None else np.ascontiguousarray(Pr, dtype=np.int64)
    ndof = _check("pgfem_generate_dof_ids", lib().pgfem_generate_dof_ids(
        nn, conn.shape[0], conn.shape[1], _ptr(conn), _ptr(Pr), _ptr(ids)))
    return ids, ndof


def psparse_apai(conn, ids, ndof):
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    ids = np.ascontiguousarray(ids, dtype=np.int64)
    Ap = np.zeros(ndof + 1, dtype=np.int32)
    nnz = _check("pgfem_psparse_apai", lib().pgfem_psparse_apai(
        conn.shape[0], conn.shape[1], _ptr(conn), _ptr(ids), ndof, _ptr(Ap), None))
    Ai = np.zeros(max(nnz, 1), dtype=np.int32)
    _check("pgfem_psparse_apai", lib().pgfem_psparse_apai(
        conn.shape[0], conn.shape[1], _ptr(conn), _ptr(ids), ndof, _ptr(Ap), _ptr(Ai)))
    return Ap, Ai[:nnz]


def state_size(model):
    return lib().pgfem_gpu_state_size(model)


# -------------------------------------------------------------- context ----
class Context:
    """Device-resident assembly context (pgfem_gpu_create / _destroy)."""

    def __init__(self, X, conn, ids, ndof, Ap, Ai, mat, npres=0, F0=None, R_cp=None):
        self._keep = dict(X=np.ascontiguousarray(X, dtype=np.float64),
                          conn=np.ascontiguousarray(conn, dtype=np.int32),
                          ids=np.ascontiguousarray(ids, dtype=np.int64),
                          Ap=np.ascontiguousarray(Ap, dtype=np.int32),
                          Ai=np.ascontiguousarray(Ai, dtype=np.int32),
                          F0=None if F0 is None else np.ascontiguousarray(F0, dtype=np.float64).reshape(9),
                          R_cp=None if R_cp is None else np.ascontiguousarray(R_cp, dtype=np.float64))
        k = self._keep
        dp = C.POINTER(C.c_double)
        self.mesh = MeshDesc(k["X"].shape[0], k["conn"].shape[0], k["conn"].shape[1],
                             k["X"].ctypes.data_as(dp), k["conn"].ctypes.data_as(C.POINTER(C.c_int)),
                             k["ids"].ctypes.data_as(C.POINTER(C.c_long)), ndof, npres,
                             None if k["F0"] is None else k["F0"].ctypes.data_as(dp),
                             None if k["R_cp"] is None else k["R_cp"].ctypes.data_as(dp))
        self.mat = mat
        self.ndof = ndof
        self.npres = npres
        self.nne = k["conn"].shape[1]
        self.ne = k["conn"].shape[0]
        self.nint = 4 if self.nne == 10 else 1
        self.ns = state_size(mat.model)
        h = C.c_void_p()
        _check("pgfem_gpu_create", lib().pgfem_gpu_create(C.byref(self.mesh), C.byref(self.mat), _ptr(k["Ap"]),
                                                          _ptr(k["Ai"]), ndof, C.byref(h)))
        self.h = h
        self.nnz = lib().pgfem_gpu_nnz(h)

    def close(self):
        if self.h:
            lib().pgfem_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_wait_test(self, limit_s, stall_next=False):
        """Failure-path tests: hand-off wait bound (s) of the linear-tet R+K
        kernel; stall_next withholds the next assembly's first hand-off."""
        _check("pgfem_gpu_set_wait_test", lib().pgfem_gpu_set_wait_test(self.h, limit_s, int(stall_next)))

    def set_neumann(self, elem, face, feature, load_type, load_np1):
        """Surface loads (the reference's NBC features, src/fd_residuals.cc:123-273):
        face k is local face face[k] (0..3) of element elem[k] with feature
        feature[k]; feature f has load_type[f] values (1 pressure, 2..3 traction)
        in load_np1[f] (3 each).  Empty elem clears."""
        el = np.ascontiguousarray(elem, dtype=np.int64).ravel()
        fc = np.ascontiguousarray(face, dtype=np.int32).ravel()
        ft = np.ascontiguousarray(feature, dtype=np.int32).ravel()
        lt = np.ascontiguousarray(load_type, dtype=np.int32).ravel()
        ld = np.ascontiguousarray(np.reshape(load_np1, (-1, 3)) if len(lt) else np.zeros((0, 3)),
                                  dtype=np.float64)
        if not (len(el) == len(fc) == len(ft)) or len(ld) != len(lt):
            raise ValueError("set_neumann: array lengths differ")
        self._nbc_keep = (el, fc, ft, lt, ld)
        _check("pgfem_gpu_set_neumann", lib().pgfem_gpu_set_neumann(self.h, len(el), _ptr(el), _ptr(fc), _ptr(ft),
                                                                      len(lt), _ptr(lt), _ptr(ld)))

    def set_neumann_loads(self, load_np1):
        ld = np.ascontiguousarray(np.reshape(load_np1, (-1, 3)), dtype=np.float64)
        _check("pgfem_gpu_set_neumann_loads", lib().pgfem_gpu_set_neumann_loads(self.h, len(ld), _ptr(ld)))

    def set_neumann_load_history(self, load_n, load_nm1):
        """The features' load values at t_n and t_{n-1} (the transient call)."""
        a = np.ascontiguousarray(np.reshape(load_n, (-1, 3)), dtype=np.float64)
        b = np.ascontiguousarray(np.reshape(load_nm1, (-1, 3)), dtype=np.float64)
        _check("pgfem_gpu_set_neumann_load_history",
               lib().pgfem_gpu_set_neumann_load_history(self.h, len(a), _ptr(a), _ptr(b)))

    def set_three_field(self, P, theta):
        """Three-field (CM3F) element: pressure P and volume theta per element
        (element order); None, None switches back to the one-field element."""
        if P is None and theta is None:
            _check("pgfem_gpu_set_three_field", lib().pgfem_gpu_set_three_field(self.h, None, None))
            return
        P = np.ascontiguousarray(P, dtype=np.float64)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        if P.shape != (self.ne,) or theta.shape != (self.ne,):
            raise ValueError("P and theta need one value per element")
        _check("pgfem_gpu_set_three_field", lib().pgfem_gpu_set_three_field(self.h, _ptr(P), _ptr(theta)))

    def get_three_field(self):
        P, theta = np.zeros(self.ne), np.zeros(self.ne)
        _check("pgfem_gpu_get_three_field", lib().pgfem_gpu_get_three_field(self.h, _ptr(P), _ptr(theta)))
        return P, theta

    def three_field_enabled(self):
        return bool(lib().pgfem_gpu_three_field_enabled(self.h))

    def three_field_increments(self, u, du, u_presc=None):
        """Element pressure / volume increments (dP, dtheta) after the
        displacement increment du, from the blocks at u."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        du = np.ascontiguousarray(du, dtype=np.float64)
        dP, dth = np.zeros(self.ne), np.zeros(self.ne)
        st = Status()
        _check("pgfem_gpu_three_field_increments", lib().pgfem_gpu_three_field_increments(
            self.h, _ptr(u), _ptr(self._presc(u_presc)), _ptr(du), _ptr(dP), _ptr(dth), C.byref(st)))
        return dP, dth, st

    def set_three_field_history(self, P_n, theta_n, P_nm1, theta_nm1):
        """Three-field P and theta per element at t_n and t_{n-1} (the
        transient element's mid points)."""
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (P_n, theta_n, P_nm1, theta_nm1)]
        _check("pgfem_gpu_set_three_field_history", lib().pgfem_gpu_set_three_field_history(
            self.h, *[_ptr(x) for x in a]))

    def three_field_increments_transient(self, u_np1, u_n, u_nm1, du, alpha, dt_np1, dt_n,
                                         presc=(None, None, None)):
        """Transient three-field local update: (dP, dtheta, Status) after the
        displacement increment du."""
        us = [np.ascontiguousarray(v, dtype=np.float64) for v in (u_np1, u_n, u_nm1, du)]
        ps = [self._presc(v) for v in presc]
        dP, dth = np.zeros(self.ne), np.zeros(self.ne)
        st = Status()
        _check("pgfem_gpu_three_field_increments_transient", lib().pgfem_gpu_three_field_increments_transient(
            self.h, *[_ptr(v) for v in us[:3]], *[_ptr(v) for v in ps], _ptr(us[3]), alpha, dt_np1, dt_n,
            _ptr(dP), _ptr(dth), C.byref(st)))
        return dP, dth, st

    def set_scatter_mode(self, mode):
        _check("pgfem_gpu_set_scatter_mode", lib().pgfem_gpu_set_scatter_mode(self.h, mode))

    def device_bytes(self):
        return lib().pgfem_gpu_device_bytes(self.h)

    def launches_per_assembly(self):
        return lib().pgfem_gpu_launches_per_assembly(self.h)

    def set_state(self, state):
        state = np.ascontiguousarray(state, dtype=np.float64)
        _check("pgfem_gpu_set_state", lib().pgfem_gpu_set_state(self.h, _ptr(state)))

    def set_state_nm1(self, state):
        """Crystal plasticity: the state at t_{n-1} (the transient element's older
        mid point); set_state sets it to the given state as well."""
        state = np.ascontiguousarray(state, dtype=np.float64)
        _check("pgfem_gpu_set_state_nm1", lib().pgfem_gpu_set_state_nm1(self.h, _ptr(state)))

    def get_state(self, level=1):
        """level 0: t_n, 1: t_{n+1}, 2: t_{n-1} (crystal plasticity)."""
        out = np.zeros((self.ne * self.nint, max(self.ns, 1)))
        _check("pgfem_gpu_get_state", lib().pgfem_gpu_get_state(self.h, level, _ptr(out)))
        return out

    def commit_state(self):
        _check("pgfem_gpu_commit_state", lib().pgfem_gpu_commit_state(self.h))

    def reset_state(self):
        _check("pgfem_gpu_reset_state", lib().pgfem_gpu_reset_state(self.h))

    def _presc(self, u_presc):
        if self.npres == 0:
            return None
        return np.ascontiguousarray(u_presc, dtype=np.float64)

    def assemble_R(self, u, u_presc=None, dt=0.0):
        u = np.ascontiguousarray(u, dtype=np.float64)
        R = np.zeros(self.ndof)
        st = Status()
        _check("pgfem_gpu_assemble_R", lib().pgfem_gpu_assemble_R(
            self.h, _ptr(u), _ptr(self._presc(u_presc)), dt, _ptr(R), C.byref(st)))
        return R, st

    def assemble_RK(self, u, u_presc=None, dt=0.0, R=None, K=None):
        u = np.ascontiguousarray(u, dtype=np.float64)
        R = np.zeros(self.ndof) if R is None else R
        K = np.zeros(self.nnz) if K is None else K
        st = Status()
        _check("pgfem_gpu_assemble_RK", lib().pgfem_gpu_assemble_RK(
            self.h, _ptr(u), _ptr(self._presc(u_presc)), dt, _ptr(R), _ptr(K), C.byref(st)))
        return R, K, st

    def assemble_RK_transient(self, u_np1, u_n, u_nm1, alpha, dt_np1, dt_n, rho, presc=(None, None, None),
                              want_K=True):
        """Transient (mid-point rule) R and K of a hyperelastic or
        crystal-plasticity context (pgfem_gpu_assemble_RK_transient); presc =
        prescribed values at t_{n+1}, t_n, t_{n-1}.  Crystal plasticity reads
        the context's states at t_{n-1} and t_n and writes the state at
        t_{n+1}.  Returns (R, K or None, Status)."""
        us = [np.ascontiguousarray(v, dtype=np.float64) for v in (u_np1, u_n, u_nm1)]
        ps = [self._presc(v) for v in presc]
        R = np.zeros(self.ndof)
        K = np.zeros(self.nnz) if want_K else None
        st = Status()
        _check("pgfem_gpu_assemble_RK_transient", lib().pgfem_gpu_assemble_RK_transient(
            self.h, *[_ptr(v) for v in us], *[_ptr(v) for v in ps], alpha, dt_np1, dt_n, rho, _ptr(R), _ptr(K),
            C.byref(st)))
        return R, K, st

    def assemble_RK_transient_device(self, d_us, d_ps, alpha, dt_np1, dt_n, rho, d_R, d_K, stream):
        """Device pointers (ints): d_us, d_ps at t_{n+1}, t_n, t_{n-1} (d_ps
        entries 0 without prescribed values), d_R, d_K (0: residual only) and a
        cudaStream_t handle (int)."""
        _check("pgfem_gpu_assemble_RK_transient_device", lib().pgfem_gpu_assemble_RK_transient_device(
            self.h, *d_us, *d_ps, alpha, dt_np1, dt_n, rho, d_R, d_K or None, stream))

    def assemble_RK_device(self, d_u, d_presc, d_R, d_K, stream, dt=0.0):
        """Device pointers (ints) and a cudaStream_t handle (int)."""
        _check("pgfem_gpu_assemble_RK_device", lib().pgfem_gpu_assemble_RK_device(
            self.h, d_u, d_presc, dt, d_R, d_K, stream))

    def set_timing(self, on=True):
        _check("pgfem_gpu_set_timing", lib().pgfem_gpu_set_timing(self.h, int(on)))

    def kernel_time(self, reset=True):
        ms = C.c_double()
        n = C.c_long()
        _check("pgfem_gpu_kernel_time", lib().pgfem_gpu_kernel_time(self.h, C.byref(ms), C.byref(n), int(reset)))
        return ms.value, n.value

    def set_cp_guess(self, guess):
        g = None if guess is None else np.ascontiguousarray(guess, dtype=np.float64)
        _check("pgfem_gpu_set_cp_guess", lib().pgfem_gpu_set_cp_guess(self.h, _ptr(g)))

    def cp_iterations(self, want_slip=False):
        it = np.zeros(self.ne * self.nint, dtype=np.int32)
        dg = np.zeros((self.ne * self.nint, 12)) if want_slip else None
        _check("pgfem_gpu_get_cp_iterations", lib().pgfem_gpu_get_cp_iterations(self.h, _ptr(it), _ptr(dg)))
        return (it, dg) if want_slip else it

    def set_cp_warm_limit(self, k):
        _check("pgfem_gpu_set_cp_warm_limit", lib().pgfem_gpu_set_cp_warm_limit(self.h, int(k)))

    def set_cp_surrogate(self, mlp):
        self._net = mlp  # keep the network alive while attached
        _check("pgfem_gpu_set_cp_surrogate", lib().pgfem_gpu_set_cp_surrogate(self.h, None if mlp is None else mlp.h))

    def cp_training_pairs(self, d_x, d_t):
        _check("pgfem_gpu_cp_training_pairs", lib().pgfem_gpu_cp_training_pairs(self.h, d_x, d_t))

    def cp_fallbacks(self):
        n = C.c_long()
        _check("pgfem_gpu_get_cp_fallbacks", lib().pgfem_gpu_get_cp_fallbacks(self.h, C.byref(n)))
        return n.value

    def set_mesh_groups(self, elem_off, F0):
        eo = np.ascontiguousarray(elem_off, dtype=np.int64)
        f0 = np.ascontiguousarray(F0, dtype=np.float64).reshape(-1, 9)
        assert len(eo) == len(f0) + 1
        _check("pgfem_gpu_set_mesh_groups", lib().pgfem_gpu_set_mesh_groups(self.h, len(f0), _ptr(eo), _ptr(f0)))

    def set_schedule(self, elems_per_block=0, grab=0):
        _check("pgfem_gpu_set_schedule", lib().pgfem_gpu_set_schedule(self.h, elems_per_block, grab))

    def schedule(self):
        e, g = C.c_int(), C.c_int()
        _check("pgfem_gpu_get_schedule", lib().pgfem_gpu_get_schedule(self.h, C.byref(e), C.byref(g)))
        return e.value, g.value

    def graph_create(self, d_u, d_presc, d_R, d_K, dt=0.0):
        """CUDA graph of one R+K assembly on device buffers (raw addresses)."""
        g = C.c_void_p()
        _check("pgfem_gpu_graph_create", lib().pgfem_gpu_graph_create(self.h, d_u, d_presc, dt, d_R, d_K,
                                                                      C.byref(g)))
        return Graph(g)

    def autotune(self, d_u, d_presc, d_R, d_K, reps=3, dt=0.0):
        e, g, ms = C.c_int(), C.c_int(), C.c_double()
        _check("pgfem_gpu_autotune", lib().pgfem_gpu_autotune(self.h, d_u, d_presc, dt, d_R, d_K, reps, C.byref(e),
                                                              C.byref(g), C.byref(ms)))
        return e.value, g.value, ms.value

    def read_status(self, clear=False):
        st = Status()
        _check("pgfem_gpu_read_status", lib().pgfem_gpu_read_status(self.h, C.byref(st), int(clear)))
        return st

    def stiffmatel_fd(self, elems, u, u_presc=None, dt=0.0):
        elems = np.ascontiguousarray(elems, dtype=np.int64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        nd = self.nne * 3
        lk = np.zeros((len(elems), nd, nd))
        fe = np.zeros((len(elems), nd))
        st = Status()
        _check("pgfem_gpu_stiffmatel_fd", lib().pgfem_gpu_stiffmatel_fd(
            self.h, len(elems), _ptr(elems), _ptr(u), _ptr(self._presc(u_presc)), dt, _ptr(lk), _ptr(fe),
            C.byref(st)))
        return lk, fe, st

    def resid_on_elem(self, elems, u, u_presc=None, dt=0.0):
        elems = np.ascontiguousarray(elems, dtype=np.int64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        fe = np.zeros((len(elems), self.nne * 3))
        st = Status()
        _check("pgfem_gpu_resid_on_elem", lib().pgfem_gpu_resid_on_elem(
            self.h, len(elems), _ptr(elems), _ptr(u), _ptr(self._presc(u_presc)), dt, _ptr(fe), C.byref(st)))
        return fe, st


def binary_version():
    """Compute capability the library's kernels were built for (100 = sm_100a)."""
    v = C.c_int(0)
    _check("pgfem_gpu_binary_version", lib().pgfem_gpu_binary_version(C.byref(v)))
    return v.value


def fp64_peak_tflops():
    t = C.c_double()
    _check("pgfem_gpu_fp64_peak", lib().pgfem_gpu_fp64_peak(C.byref(t)))
    return t.value


def cm_integrate(mat, F, state_n=None, dt=0.0, want_L=True):
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(-1, 9)
    nqp = F.shape[0]
    ns = state_size(mat.model)
    S = np.zeros((nqp, 9))
    L = np.zeros((nqp, 81)) if want_L else None
    snp1 = np.zeros((nqp, max(ns, 1)))
    sn = None if state_n is None else np.ascontiguousarray(state_n, dtype=np.float64)
    qst = np.zeros(nqp, dtype=np.int32)
    _check("pgfem_gpu_cm_integrate", lib().pgfem_gpu_cm_integrate(
        C.byref(mat), nqp, _ptr(F), dt, None, _ptr(sn), _ptr(snp1), _ptr(S), _ptr(L), _ptr(qst)))
    return S, L, snp1, qst


CP_NOALLOC_MAX_POINTS = 4096


def cp_integrate_noalloc(mat, nqp, d_F, d_R_cp, d_state_n, dt, d_state_np1, d_dgam=None, d_iters=None,
                         stream=None, want_status=True):
    """CP point update on caller-owned device buffers (raw device addresses as ints,
    component-major layouts) through pgfem_gpu_cp_integrate_noalloc, which allocates
    no device memory.  Returns the failure counts (the call then waits for the
    stream) or None when want_status is False (the call stays asynchronous)."""
    st = Status() if want_status else None
    _check("pgfem_gpu_cp_integrate_noalloc", lib().pgfem_gpu_cp_integrate_noalloc(
        C.byref(mat), nqp, d_F, d_R_cp, d_state_n, dt, d_state_np1, d_dgam, d_iters,
        C.byref(st) if st is not None else None, stream))
    return st


# ------------------------------------------------------- warm-start network --
MLP_IN, MLP_OUT = 34, 12


class MlpTrainOpts(C.Structure):
    _fields_ = [("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_float), ("lr_min", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float), ("seed", C.c_ulonglong)]


class Mlp:
    """The warm-start network of the CP local Newton (pgfem_mlp_* entry points)."""

    def __init__(self, seed=0):
        h = C.c_void_p()
        _check("pgfem_mlp_create", lib().pgfem_mlp_create(seed, C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pgfem_mlp_destroy(self.h)
            self.h = None

    @staticmethod
    def num_params():
        return lib().pgfem_mlp_num_params()

    def params(self):
        p = np.zeros(self.num_params(), dtype=np.float32)
        _check("pgfem_mlp_get_params", lib().pgfem_mlp_get_params(self.h, _ptr(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.num_params()
        _check("pgfem_mlp_set_params", lib().pgfem_mlp_set_params(self.h, _ptr(p)))

    def set_wait_test(self, limit_s, stall_next=False):
        """Failure-path tests: tensor-core completion wait bound (s); stall_next
        withholds the next forward pass's first MMA chain per CTA."""
        _check("pgfem_mlp_set_wait_test", lib().pgfem_mlp_set_wait_test(self.h, limit_s, int(stall_next)))

    def set_scaling(self, x_mean, x_std, y_std):
        a = [np.ascontiguousarray(v, dtype=np.float32) for v in (x_mean, x_std, y_std)]
        _check("pgfem_mlp_set_scaling", lib().pgfem_mlp_set_scaling(self.h, *[_ptr(v) for v in a]))

    def scaling(self):
        xm, xi, ys = np.zeros(MLP_IN, np.float32), np.zeros(MLP_IN, np.float32), np.zeros(MLP_OUT, np.float32)
        _check("pgfem_mlp_get_scaling", lib().pgfem_mlp_get_scaling(self.h, _ptr(xm), _ptr(xi), _ptr(ys)))
        return xm, xi, ys

    def fit_scaling(self, n, d_x, d_t):
        _check("pgfem_mlp_fit_scaling", lib().pgfem_mlp_fit_scaling(self.h, n, d_x, d_t))

    def predict(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, MLP_IN)
        y = np.zeros((x.shape[0], MLP_OUT), dtype=np.float32)
        _check("pgfem_mlp_predict", lib().pgfem_mlp_predict(self.h, x.shape[0], _ptr(x), _ptr(y)))
        return y

    def predict_device(self, n, d_x, d_y, stream=None):
        _check("pgfem_mlp_predict_device", lib().pgfem_mlp_predict_device(self.h, n, d_x, d_y, stream))

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, MLP_IN)
        t = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, MLP_OUT)
        g = np.zeros(self.num_params(), dtype=np.float32)
        loss = C.c_double()
        _check("pgfem_mlp_loss_grad", lib().pgfem_mlp_loss_grad(self.h, x.shape[0], _ptr(x), _ptr(t), _ptr(g),
                                                                C.byref(loss)))
        return loss.value, g

    def train_device(self, n, d_x, d_t, epochs=10, batch=4096, lr=2e-3, lr_min=5e-5, beta1=0.9, beta2=0.999,
                     eps=1e-8, seed=0):
        o = MlpTrainOpts(epochs, batch, lr, lr_min, beta1, beta2, eps, seed)
        hist = np.zeros(max(epochs, 1))
        _check("pgfem_mlp_train_device", lib().pgfem_mlp_train_device(self.h, n, d_x, d_t, C.byref(o),
                                                                      _ptr(hist)))
        return hist[:epochs]


class Graph:
    """A captured assembly (pgfem_gpu_graph_*)."""

    def __init__(self, h):
        self.h = h

    def launch(self, stream=None):
        _check("pgfem_gpu_graph_launch", lib().pgfem_gpu_graph_launch(self.h, stream))

    def destroy(self):
        if self.h:
            lib().pgfem_gpu_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pgfem_gpu_graph_destroy(self.h)
            self.h = None


# ---- linear solve and Newton-Raphson --------------------------------------
SOLVER_GMRES, SOLVER_BCG_STAB = 0, 1
PRECOND_NONE, PRECOND_DIAG_SCALE = 4, 5
GMRES_MAX_KDIM = 1000
NEWTON_HISTORY = 32


class SolverOpts(C.Structure):
    _fields_ = [("solver", C.c_int), ("precond", C.c_int), ("maxit", C.c_int), ("kdim", C.c_int),
                ("tol", C.c_double), ("check_every", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("iters", C.c_int), ("res_norm", C.c_double), ("converged", C.c_int), ("breakdown", C.c_int)]


class NewtonOpts(C.Structure):
    _fields_ = [("iter_max", C.c_int), ("nor_min", C.c_double), ("computer_zero", C.c_double)]


class NewtonInfo(C.Structure):
    _fields_ = [("iters", C.c_int), ("converged", C.c_int), ("lin_iters", C.c_int), ("lin_failed", C.c_int),
                ("elem_failures", C.c_long), ("nor", C.c_double), ("nor2", C.c_double),
                ("nor_hist", C.c_double * NEWTON_HISTORY)]

    def history(self):
        return [self.nor_hist[i] for i in range(min(self.iters + 1, NEWTON_HISTORY))]


class Solver:
    """Device linear solver over one CSR pattern (pgfem_gpu_solver_*)."""

    def __init__(self, Ap, Ai, nrows, solver=SOLVER_GMRES, precond=PRECOND_DIAG_SCALE, maxit=5000, kdim=100,
                 tol=1e-10, check_every=8):
        self._Ap = np.ascontiguousarray(Ap, dtype=np.int32)
        self._Ai = np.ascontiguousarray(Ai, dtype=np.int32)
        self.n = int(nrows)
        self.nnz = int(self._Ap[-1])
        self.opts = SolverOpts(solver, precond, maxit, kdim, tol, check_every)
        h = C.c_void_p()
        _check("pgfem_gpu_solver_create", lib().pgfem_gpu_solver_create(_ptr(self._Ap), _ptr(self._Ai), self.n,
                                                                        C.byref(self.opts), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().pgfem_gpu_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_bytes(self):
        return lib().pgfem_gpu_solver_device_bytes(self.h)

    def spmv(self, d_K, d_x, d_y, stream=None):
        _check("pgfem_gpu_spmv", lib().pgfem_gpu_spmv(self.h, d_K, d_x, d_y, stream))

    def solve(self, d_K, d_b, d_x, stream=None):
        info = SolveInfo()
        _check("pgfem_gpu_solve", lib().pgfem_gpu_solve(self.h, d_K, d_b, d_x, C.byref(info), stream))
        return info

    def newton_step(self, ctx, d_u, d_presc=None, dt=0.0, iter_max=10, nor_min=1e-10, computer_zero=1e-15,
                    stream=None):
        o = NewtonOpts(iter_max, nor_min, computer_zero)
        info = NewtonInfo()
        _check("pgfem_gpu_newton_step", lib().pgfem_gpu_newton_step(ctx.h, self.h, d_u, d_presc, dt, C.byref(o),
                                                                    C.byref(info), stream))
        return info


# ------------------------------------------------------------ input files ----
class InputInfo(C.Structure):
    _fields_ = [("nn", C.c_long), ("ne", C.c_long), ("nne", C.c_int), ("npres", C.c_long), ("nmat", C.c_int),
                ("nconc", C.c_long), ("norient", C.c_long), ("lin_maxit", C.c_long), ("lin_err", C.c_double),
                ("lim_zero", C.c_double), ("nln", C.c_long), ("nel_s", C.c_long), ("nel_v", C.c_long),
                ("nperiodic", C.c_long)]


class SolverFile(C.Structure):
    _fields_ = [("nor_min", C.c_double), ("iter_max", C.c_long), ("npres", C.c_long), ("FNR", C.c_long),
                ("dAL0", C.c_double), ("dALMAX", C.c_double), ("physicsno", C.c_int),
                ("max_NR_staggering", C.c_int), ("max_subdivision", C.c_int), ("nt", C.c_long),
                ("n_print", C.c_long), ("n_load", C.c_long), ("n_incr", C.c_long)]


class ModelParams(C.Structure):
    _fields_ = [("mat_id", C.c_int), ("model_type", C.c_int), ("uq", C.c_int), ("np", C.c_int),
                ("p", C.c_double * 16), ("unit_cell", C.c_int), ("ort_option", C.c_int * 3),
                ("ort_file", C.c_char * 256), ("ort_angles", C.c_double * 3), ("solver_set", C.c_int),
                ("max_itr_stag", C.c_int), ("max_itr_hardening", C.c_int), ("max_itr_M", C.c_int),
                ("max_subdivision", C.c_int), ("tol_hardening", C.c_double), ("tol_M", C.c_double),
                ("computer_zero", C.c_double)]


CM_HYPER_ELASTICITY, CM_CRYSTAL_PLASTICITY, CM_J2_PLASTICITY_DAMAGE = 0, 1, 4


def _check_input(fn, r):
    if r < 0:
        e = PgfemError(fn, r)
        e.args = (e.args[0] + ": " + lib().pgfem_input_last_error().decode(),)
        raise e
    return r


class InputMesh:
    """A PGFem3D mesh read from its <base><r>.in files (pgfem_input_read_mesh),
    partitions merged: X (nn,3), conn (ne,nne), codes (nn,3) support codes,
    defl (npres,), per-element material / partition data, material lines."""

    def __init__(self, base, nparts=1, bc_base=None, physics=None):
        """bc_base: supports and prescribed values from <bc_base>_<r>.bc and
        <bc_base>.bcv (a BC directory) instead of the mesh files.  physics:
        (ids, ndim) of a multiphysics mesh (read_multiphysics); the mechanical
        supports section (id 0) is kept."""
        h = C.c_void_p()
        bc = None if bc_base is None else bc_base.encode()
        if physics is None:
            _check_input("pgfem_input_read_mesh", lib().pgfem_input_read_mesh_bc(base.encode(), nparts, bc, C.byref(h)))
        else:
            ids, nd = physics
            nd = np.ascontiguousarray(nd, dtype=np.int32)
            _check_input("pgfem_input_read_mesh", lib().pgfem_input_read_mesh_mp(
                base.encode(), nparts, bc, len(nd), _ptr(nd), list(ids).index(0), C.byref(h)))
        try:
            info = InputInfo()
            _check("pgfem_input_get_info", lib().pgfem_input_get_info(h, C.byref(info)))
            self.info = info
            nn, ne, nne = info.nn, info.ne, info.nne
            self.X = np.zeros((nn, 3))
            self.conn = np.zeros((ne, nne), dtype=np.int32)
            self.codes = np.zeros((nn, 3), dtype=np.int64)
            self.defl = np.zeros(info.npres)
            _check("pgfem_input_get_mesh", lib().pgfem_input_get_mesh(h, _ptr(self.X), _ptr(self.conn),
                                                                      _ptr(self.codes), _ptr(self.defl)))
            self.elem_mat = np.zeros((ne, 2), dtype=np.int64)
            self.elem_hom = np.zeros((ne, 2), dtype=np.int64)
            self.elem_part = np.zeros(ne, dtype=np.int32)
            self.elem_local = np.zeros(ne, dtype=np.int64)
            _check("pgfem_input_get_elements", lib().pgfem_input_get_elements(
                h, _ptr(self.elem_mat), _ptr(self.elem_hom), _ptr(self.elem_part), _ptr(self.elem_local)))
            self.Pr = np.zeros(nn, dtype=np.int64)
            _check("pgfem_input_get_periodic", lib().pgfem_input_get_periodic(h, _ptr(self.Pr)))
            self.materials = np.zeros((info.nmat, 13))
            self.dev_pot = np.zeros(info.nmat, dtype=np.int32)
            self.vol_pot = np.zeros(info.nmat, dtype=np.int32)
            _check("pgfem_input_get_materials", lib().pgfem_input_get_materials(
                h, _ptr(self.materials), _ptr(self.dev_pot), _ptr(self.vol_pot)))
            self._h = h
        except Exception:
            lib().pgfem_input_destroy(h)
            raise

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.pgfem_input_destroy(self._h)
            self._h = None

    def partition(self, part):
        """(node_map (merged id of each local node), first element, element count) of a partition."""
        nn, ne = C.c_long(), C.c_long()
        _check("pgfem_input_get_partition", lib().pgfem_input_get_partition(self._h, part, C.byref(nn), C.byref(ne),
                                                                          None))
        nm = np.zeros(nn.value, dtype=np.int64)
        _check("pgfem_input_get_partition", lib().pgfem_input_get_partition(self._h, part, None, None, _ptr(nm)))
        e0 = int(np.searchsorted(self.elem_part, part))
        return nm, e0, ne.value

    def orientations(self, base):
        """(angles (ne,3), EulerAngleType) from <base>_<r>.in."""
        a = np.zeros((self.info.ne, 3))
        et = C.c_int()
        _check_input("pgfem_input_read_orientations",
                     lib().pgfem_input_read_orientations(self._h, base.encode(), _ptr(a), C.byref(et)))
        return a, et.value

    def material(self, imat=0, model=MODEL_HE, **kw):
        """pgfem_material_desc from material line imat: E = Ex, nu = nyz (the
        isotropic entries), dev_pot = devPotFlag for HE, vol_pot = volPotFlag
        for HE and J2; keywords add or override fields (J2 / CP parameters)."""
        m = self.materials[imat]
        args = dict(E=m[0], nu=m[6])
        if model == MODEL_HE:
            args["dev_pot"] = int(self.dev_pot[imat])
        if model in (MODEL_HE, MODEL_J2) and int(self.vol_pot[imat]) in (2, 3):
            args["vol_pot"] = int(self.vol_pot[imat])
        args.update(kw)
        return material(model, **args)

    def element_faces(self):
        """(bnd_type, bnd_id), each (ne, 4): the boundary feature of every face."""
        bt = np.zeros((self.info.ne, 4), dtype=np.int32)
        bi = np.zeros((self.info.ne, 4), dtype=np.int32)
        _check("pgfem_input_get_element_faces", lib().pgfem_input_get_element_faces(self._h, _ptr(bt), _ptr(bi)))
        return bt, bi

    def dof_setup(self):
        """(ids, ndof, Ap, Ai) of the merged mesh (generate_dof_ids with the
        periodic links + Psparse_ApAi)."""
        Pr = self.Pr if self.info.nperiodic else None
        ids, ndof = generate_dof_ids(self.conn, self.X.shape[0], self.codes, Pr)
        Ap, Ai = psparse_apai(self.conn, ids, ndof)
        return ids, ndof, Ap, Ai


class NbcFile:
    """Surface loads of <ipath>/NBC/<physics>.nbc (pgfem_input_read_nbc):
    features (type, id, load type), the loaded faces of a mesh and the load
    values at a time -- the inputs of Context.set_neumann / set_neumann_loads."""

    def __init__(self, ipath, physics="Mechanical"):
        h = C.c_void_p()
        _check_input("pgfem_input_read_nbc", lib().pgfem_input_read_nbc(ipath.encode(), physics.encode(), C.byref(h)))
        self._h = h
        n = C.c_int()
        _check("pgfem_nbc_get_features", lib().pgfem_nbc_get_features(h, C.byref(n), None, None, None))
        self.ftype = np.zeros(n.value, dtype=np.int32)
        self.fid = np.zeros(n.value, dtype=np.int32)
        self.load_type = np.zeros(n.value, dtype=np.int32)
        _check("pgfem_nbc_get_features", lib().pgfem_nbc_get_features(h, None, _ptr(self.ftype), _ptr(self.fid),
                                                                      _ptr(self.load_type)))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.pgfem_nbc_destroy(self._h)
            self._h = None

    def faces(self, mesh):
        """(elem, face, feature) of the faces of an InputMesh these features load."""
        n = C.c_long()
        _check("pgfem_nbc_faces", lib().pgfem_nbc_faces(self._h, mesh._h, C.byref(n), None, None, None))
        el = np.zeros(n.value, dtype=np.int64)
        fc = np.zeros(n.value, dtype=np.int32)
        ft = np.zeros(n.value, dtype=np.int32)
        _check("pgfem_nbc_faces", lib().pgfem_nbc_faces(self._h, mesh._h, C.byref(n), _ptr(el), _ptr(fc), _ptr(ft)))
        return el, fc, ft

    def load_values(self, t):
        v = np.zeros((len(self.ftype), 3))
        _check_input("pgfem_nbc_load_values", lib().pgfem_nbc_load_values(self._h, t, _ptr(v)))
        return v


def cp_resolved_shear(mat, F, pF, g, R):
    """(tau, gamma_dot), each (n, 12), of crystal plasticity points in the
    order and sign of the reference's restart files (pgfem_cp_resolved_shear)."""
    F = np.ascontiguousarray(np.reshape(F, (-1, 9)), dtype=np.float64)
    pF = np.ascontiguousarray(np.reshape(pF, (-1, 9)), dtype=np.float64)
    g = np.ascontiguousarray(np.ravel(g), dtype=np.float64)
    R = np.ascontiguousarray(np.reshape(R, (-1, 9)), dtype=np.float64)
    n = len(F)
    tau, gd = np.zeros((n, 12)), np.zeros((n, 12))
    _check("pgfem_cp_resolved_shear", lib().pgfem_cp_resolved_shear(C.byref(mat), n, _ptr(F), _ptr(pF), _ptr(g),
                                                                      _ptr(R), _ptr(tau), _ptr(gd)))
    return tau, gd


def load_expression(expr, t):
    """Value of a load expression of time t (pgfem_load_expression)."""
    v = C.c_double()
    _check_input("pgfem_load_expression", lib().pgfem_load_expression(expr.encode(), t, C.byref(v)))
    return v.value


def read_multiphysics(path, max_phys=16):
    """(ids, ndim) per physics in file order (0 mechanical, 1 thermal)."""
    ids = np.zeros(max_phys, dtype=np.int32)
    nd = np.zeros(max_phys, dtype=np.int32)
    n = C.c_int()
    _check_input("pgfem_input_read_multiphysics",
                 lib().pgfem_input_read_multiphysics(path.encode(), max_phys, _ptr(ids), _ptr(nd), C.byref(n)))
    return ids[:n.value].tolist(), nd[:n.value].tolist()


def read_solver_file(path, npd=-1):
    """Returns (SolverFile, times, print_steps, load_steps, load_incr (n_load, n_incr));
    npd = the mesh's prescribed-value count (InputMesh.info.npres)."""
    sf = SolverFile()
    _check_input("pgfem_input_read_solver_file",
                 lib().pgfem_input_read_solver_file(path.encode(), npd, C.byref(sf), None, None, None, None))
    times = np.zeros(sf.nt + 1)
    ps = np.zeros(sf.n_print, dtype=np.int64)
    ls = np.zeros(sf.n_load, dtype=np.int64)
    li = np.zeros((sf.n_load, sf.n_incr))
    _check_input("pgfem_input_read_solver_file", lib().pgfem_input_read_solver_file(
        path.encode(), npd, C.byref(sf), _ptr(times), _ptr(ps), _ptr(ls), _ptr(li)))
    return sf, times, ps, ls, li


def read_model_params(path, max_entries=64):
    out = (ModelParams * max_entries)()
    n = C.c_int()
    _check_input("pgfem_input_read_model_params",
                 lib().pgfem_input_read_model_params(path.encode(), max_entries, out, C.byref(n)))
    return [out[i] for i in range(min(n.value, max_entries))]


def cp_material(mp, E, nu, cp_tol=1e-10, cp_max_iter=25):
    """pgfem_material_desc of a crystal plasticity model_params entry."""
    assert mp.model_type == CM_CRYSTAL_PLASTICITY and mp.np == 7
    p = list(mp.p)[:7]
    return material(MODEL_CP, E=E, nu=nu, gamma_dot_0=p[0], m=p[1], G0=p[2], g0=p[3], gs_0=p[4],
                    gamma_dot_s=p[5], w=p[6], cp_tol=cp_tol, cp_max_iter=cp_max_iter)


def j2_material(mp, E, nu, vol_pot=99):
    """pgfem_material_desc of a J2 model_params entry (sigma_y = k0, H = hp;
    EINVAL for beta != 0 or active damage)."""
    out = MaterialDesc()
    _check("pgfem_input_j2_material", lib().pgfem_input_j2_material(C.byref(mp), E, nu, vol_pot, C.byref(out)))
    return out


def euler_rotation(angles):
    a = np.ascontiguousarray(angles, dtype=np.float64).reshape(-1, 3)
    R = np.zeros((a.shape[0], 3, 3))
    _check("pgfem_euler_rotation", lib().pgfem_euler_rotation(a.shape[0], _ptr(a), _ptr(R)))
    return R


# --------------------------------------------------------------- restart ----
def restart_block_size(model):
    return lib().pgfem_restart_block_size(model)


def restart_format(path, model, u_nm1, u_n, blocks):
    """One rank's restart file: u_nm1, u_n nodal (nn,3); blocks (ne, n_ip, block_size)."""
    u_nm1 = np.ascontiguousarray(u_nm1, dtype=np.float64)
    u_n = np.ascontiguousarray(u_n, dtype=np.float64)
    blocks = np.ascontiguousarray(blocks, dtype=np.float64)
    _check_input("pgfem_restart_format", lib().pgfem_restart_format(
        path.encode(), u_n.shape[0], blocks.shape[0], blocks.shape[1], model, _ptr(u_nm1), _ptr(u_n), _ptr(blocks)))


def restart_parse(path, model, nn, ne, n_ip):
    bs = _check("pgfem_restart_block_size", restart_block_size(model))
    u_nm1 = np.zeros((nn, 3))
    u_n = np.zeros((nn, 3))
    blocks = np.zeros((ne, n_ip, bs))
    _check_input("pgfem_restart_parse", lib().pgfem_restart_parse(
        path.encode(), nn, ne, n_ip, model, _ptr(u_nm1), _ptr(u_n), _ptr(blocks)))
    return u_nm1, u_n, blocks


def restart_write_partitions(inp, name, step, model, u_nm1, u_n, blocks):
    """Per-partition restart files <name>_<r>_<step>.res of an InputMesh from
    merged nodal u_nm1, u_n (nn, 3) and blocks (ne, n_ip, block_size)."""
    u_nm1 = np.ascontiguousarray(u_nm1, dtype=np.float64)
    u_n = np.ascontiguousarray(u_n, dtype=np.float64)
    blocks = np.ascontiguousarray(blocks, dtype=np.float64)
    _check_input("pgfem_restart_write_partitions", lib().pgfem_restart_write_partitions(
        inp._h, name.encode(), step, model, blocks.shape[1], _ptr(u_nm1), _ptr(u_n), _ptr(blocks)))


def write_restart(ctx, path, u_nm1, u_n, presc_nm1=None, presc_n=None, state_nm1=None):
    u_nm1 = np.ascontiguousarray(u_nm1, dtype=np.float64)
    u_n = np.ascontiguousarray(u_n, dtype=np.float64)
    pn1 = None if presc_nm1 is None else np.ascontiguousarray(presc_nm1, dtype=np.float64)
    pn = None if presc_n is None else np.ascontiguousarray(presc_n, dtype=np.float64)
    sm = None if state_nm1 is None else np.ascontiguousarray(state_nm1, dtype=np.float64)
    _check_input("pgfem_gpu_write_restart", lib().pgfem_gpu_write_restart(
        ctx.h, path.encode(), _ptr(u_nm1), _ptr(u_n), _ptr(pn1), _ptr(pn), _ptr(sm)))


def read_restart(ctx, path):
    """Returns the free-DOF (u_nm1, u_n); CP contexts take the state at t_n from the file."""
    u_nm1 = np.zeros(ctx.ndof)
    u_n = np.zeros(ctx.ndof)
    _check_input("pgfem_gpu_read_restart", lib().pgfem_gpu_read_restart(ctx.h, path.encode(), _ptr(u_nm1), _ptr(u_n)))
    return u_nm1, u_n
