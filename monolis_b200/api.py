"""ctypes mirror of the monolis C API (include/monolis.h, include/monolis_b200.h).

`MonolisLib(path)` binds any shared library that exports the monolis C API;
`Monolis(lib)` owns one `MONOLIS` struct and exposes the reference's calls
under the same names and argument meaning (0-based node/dof indices, as in
the reference C wrapper `wrapper/matrix/monolis_spmat_handler_c.c`).

The product library is `monolis_b200/libmonolis_b200.so` (`load_product()`);
it fails loudly when the library is missing, there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PRODUCT_SO = os.path.join(_HERE, "libmonolis_b200.so")

# ---- constants (include/monolis.h, include/monolis_b200.h) ----
ITER_CG = 1
ITER_GROPCG = 2
ITER_PIPECG = 3
ITER_BICGSTAB = 5
ITER_BICGSTAB_N128 = 9
PREC_NONE = 0
PREC_DIAG = 1
PRM_I_METHOD = 1
PRM_I_PRECOND = 2
PRM_I_MAX_ITER = 3
PRM_I_CUR_ITER = 4
PRM_I_IERR = 5
PRM_I_IS_INIT_X = 10
PRM_I_IS_MEASUREMENT = 13
PRM_I_IS_ERROR_ABORT = 16
PRM_I_SHOW_ITERLOG = 20
PRM_I_SHOW_TIME = 21
PRM_I_SHOW_SUMMARY = 22
PRM_R_TOL = 1
PRM_R_CUR_RESID = 2
R_TIME_SOL = 3
R_TIME_PREP = 4
B200_PRM_I_PRECISION = 30
B200_PRM_I_MATRIX_CACHE = 31
B200_PRM_I_MATRIX_VERSION = 32
B200_PRM_I_N_REFINE = 33
B200_PRM_I_BATCH = 34
B200_PRM_I_CHECK = 35
B200_PRM_I_LAUNCHES = 36
B200_PRM_I_ITER_RR = 37
B200_PRM_I_UNROLL_FP64 = 38
B200_PRM_I_UNROLL_FP32 = 39
B200_PRM_I_KERNEL_TIMERS = 40
B200_PRM_I_REFRESH_PERIOD = 41
B200_PRM_I_WIDE_SLICES_FP64 = 42
B200_PRM_I_WIDE_SLICES_FP32 = 43
B200_PRM_I_WAIT_LIMIT = 44
B200_PRM_I_WAIT_DELAY_US = 45
B200_PRM_I_UNIFORM_SLICES_FP64 = 46
B200_PRM_I_UNIFORM_SLICES_FP32 = 47
B200_PRM_R_REFRESH_DELTA = 30
B200_PRM_R_TIME_H2D = 31
B200_PRM_R_TIME_D2H = 32
B200_PRM_R_TIME_LOOP = 33
B200_PRM_R_SPMV_BYTES_FP64 = 34
B200_PRM_R_SPMV_BYTES_FP32 = 35
B200_PRM_R_TIME_KERNEL = 40
STATUS_NAMES = {0: "ok", 1: "max_iter", 2: "breakdown", 3: "nonfinite", 4: "timeout", 5: "bad_input",
                6: "cuda_error"}

_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)


class MONOLIS_PRM(C.Structure):
    _fields_ = [("com_top_dir_name", C.c_char * 1024), ("com_part_dir_name", C.c_char * 1024),
                ("com_file_name", C.c_char * 1024), ("Iarray", C.c_int * 100), ("Rarray", C.c_double * 100)]


class MONOLIS_MAT_VAL_R(C.Structure):
    _fields_ = [(n, _dp) for n in ("A", "U", "D", "L", "X", "B")]


class MONOLIS_MAT_VAL_C(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("A", "U", "D", "L", "X", "B")]


class MONOLIS_MAT_SEPARATED_CSR(C.Structure):
    _fields_ = [(n, _ip) for n in ("indexU", "indexL", "itemU", "itemL")]


class MONOLIS_MAT_CSR(C.Structure):
    _fields_ = [("index", _ip), ("item", _ip)]


class MONOLIS_MAT_CSC(C.Structure):
    _fields_ = [("index", _ip), ("item", _ip), ("perm", _ip)]


class MONOLIS_MAT(C.Structure):
    _fields_ = [("N", C.c_int), ("NP", C.c_int), ("NDOF", C.c_int), ("n_dof_list", _ip), ("n_dof_index", _ip),
                ("n_dof_index2", _ip), ("R", MONOLIS_MAT_VAL_R), ("C", MONOLIS_MAT_VAL_C),
                ("SCSR", MONOLIS_MAT_SEPARATED_CSR), ("CSR", MONOLIS_MAT_CSR), ("CSC", MONOLIS_MAT_CSC)]


class MONOLIS(C.Structure):
    _fields_ = [("prm", MONOLIS_PRM), ("mat", MONOLIS_MAT), ("prec", MONOLIS_MAT)]


class MONOLIS_COM(C.Structure):
    _fields_ = [("comm", C.c_int), ("my_rank", C.c_int), ("comm_size", C.c_int), ("n_internal_vertex", C.c_int),
                ("recv_n_neib", C.c_int), ("recv_neib_pe", _ip), ("recv_index", _ip), ("recv_item", _ip),
                ("send_n_neib", C.c_int), ("send_neib_pe", _ip), ("send_index", _ip), ("send_item", _ip)]


_MP = C.POINTER(MONOLIS)
_CP = C.POINTER(MONOLIS_COM)

# name -> (restype, argtypes) for the API common to the product and the oracle
_COMMON = {
    "monolis_initialize": (None, [_MP]),
    "monolis_finalize": (None, [_MP]),
    "monolis_com_initialize_by_self": (None, [_CP]),
    "monolis_com_finalize": (None, [_CP]),
    "monolis_set_method": (None, [_MP, C.c_int]),
    "monolis_set_precond": (None, [_MP, C.c_int]),
    "monolis_set_maxiter": (None, [_MP, C.c_int]),
    "monolis_set_tolerance": (None, [_MP, C.c_double]),
    "monolis_set_init_x": (None, [_MP, C.c_bool]),
    "monolis_set_error_abort": (None, [_MP, C.c_bool]),
    "monolis_show_iterlog": (None, [_MP, C.c_bool]),
    "monolis_show_timelog": (None, [_MP, C.c_bool]),
    "monolis_show_summary": (None, [_MP, C.c_bool]),
    "monolis_get_converge_iter": (None, [_MP, _ip]),
    "monolis_get_converge_residual": (None, [_MP, _dp]),
    "monolis_get_error_tag": (None, [_MP, _ip]),
    "monolis_get_nonzero_pattern_by_simple_mesh_R": (None, [_MP, C.c_int, C.c_int, C.c_int, C.c_int,
                                                            C.POINTER(_ip)]),
    "monolis_get_nonzero_pattern_by_nodal_graph_R": (None, [_MP, C.c_int, C.c_int, _ip, _ip]),
    "monolis_add_scalar_to_sparse_matrix_R": (None, [_MP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]),
    "monolis_set_scalar_to_sparse_matrix_R": (None, [_MP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]),
    "monolis_get_scalar_from_sparse_matrix_R": (None, [_MP, C.c_int, C.c_int, C.c_int, C.c_int, _dp,
                                                       C.POINTER(C.c_bool)]),
    "monolis_add_matrix_to_sparse_matrix_R": (None, [_MP, C.c_int, _ip, C.POINTER(_dp)]),
    "monolis_set_matrix_BCSR_R": (None, [_MP, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _ip, _ip]),
    "monolis_set_Dirichlet_bc_R": (None, [_MP, _dp, C.c_int, C.c_int, C.c_double]),
    "monolis_matvec_product_R": (None, [_MP, _CP, _dp, _dp]),
    "monolis_inner_product_R": (None, [_MP, _CP, C.c_int, _dp, _dp, _dp]),
    "monolis_solve_R": (None, [_MP, _CP, _dp, _dp]),
    "monolis_get_CSC_format": (None, [C.c_int, C.c_int, C.c_int, _ip, _ip, _ip, _ip, _ip]),
}

_PRODUCT = {
    "monolis_b200_set_precision": (C.c_int, [_MP, C.c_int]),
    "monolis_b200_set_matrix_cache": (None, [_MP, C.c_bool]),
    "monolis_b200_matrix_changed": (None, [_MP]),
    "monolis_b200_get_nonzero_pattern_by_simple_mesh_flat_R": (C.c_int, [_MP, C.c_int, C.c_int, C.c_int, C.c_int,
                                                                          _ip]),
    "monolis_b200_add_elements_R": (C.c_int, [_MP, C.c_int, C.c_int, _ip, _dp, C.c_longlong, _dp]),
    "monolis_b200_stream": (C.c_void_p, []),
    "monolis_b200_device_prepare": (C.c_int, [_MP]),
    "monolis_b200_device_solve_R": (C.c_int, [_MP, C.c_void_p, C.c_void_p]),
    "monolis_b200_device_solve_com_R": (C.c_int, [_MP, _CP, C.c_void_p, C.c_void_p]),
    "monolis_b200_device_matvec_R": (C.c_int, [_MP, C.c_void_p, C.c_void_p]),
    "monolis_b200_device_matvec_R32": (C.c_int, [_MP, C.c_void_p, C.c_void_p]),
    "monolis_b200_device_info": (C.c_int, [_MP, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                           C.POINTER(C.c_int)]),
    "monolis_b200_inner_product_noalloc_R": (C.c_int, [C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p,
                                                       C.c_void_p]),
    "monolis_b200_solve_transpose_R": (C.c_int, [_MP, _CP, _dp, _dp]),
    "monolis_b200_device_solve_transpose_R": (C.c_int, [_MP, C.c_void_p, C.c_void_p]),
    "monolis_b200_matvec_transpose_R": (C.c_int, [_MP, _CP, _dp, _dp]),
    "monolis_b200_device_matvec_transpose_R": (C.c_int, [_MP, C.c_void_p, C.c_void_p]),
    "monolis_b200_sampled_outer_product_R": (C.c_int, [_MP, _dp, _dp, C.c_double, _dp]),
    "monolis_b200_device_sampled_outer_product_R": (C.c_int, [_MP, C.c_void_p, C.c_void_p, C.c_double,
                                                              C.c_void_p]),
    "monolis_b200_element_gradient_R": (C.c_int, [_MP, C.c_int, C.c_int, _ip, _dp, C.c_longlong, _dp, _dp, _ip,
                                                  C.c_double, _dp]),
    "monolis_b200_device_element_gradient_R": (C.c_int, [_MP, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                                         C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p,
                                                         C.c_double, C.c_void_p]),
    "monolis_b200_batch_create": (C.c_int, [C.POINTER(C.c_void_p)]),
    "monolis_b200_batch_destroy": (None, [C.c_void_p]),
    "monolis_b200_batch_add_system": (C.c_int, [C.c_void_p, _MP]),
    "monolis_b200_batch_add_csr": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _ip, _ip, _dp]),
    "monolis_b200_batch_prepare": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "monolis_b200_batch_set_config": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_longlong]),
    "monolis_b200_batch_get_config": (C.c_int, [C.c_void_p, _ip, _ip, C.POINTER(C.c_longlong)]),
    "monolis_b200_batch_get_unroll": (C.c_int, [C.c_void_p, _ip]),
    "monolis_b200_batch_autotune": (C.c_int, [C.c_void_p, C.c_int, _ip, _ip, _ip, C.POINTER(C.c_longlong), _dp]),
    "monolis_b200_batch_solve_R": (C.c_int, [C.c_void_p, C.POINTER(_dp), C.POINTER(_dp), C.c_double, C.c_int,
                                             C.c_int, _ip, _dp, _ip]),
    "monolis_b200_batch_info": (C.c_int, [C.c_void_p, _ip, C.POINTER(C.c_longlong)]),
    "monolis_b200_batch_device_vectors": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "monolis_b200_batch_device_solve_R": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int, _ip, _dp, _ip]),
    "monolis_b200_batch_last_seconds": (C.c_double, [C.c_void_p]),
    "monolis_b200_solve_multi_R": (C.c_int, [_MP, _CP, C.c_int, _dp, _dp, _ip, _dp, _ip]),
    "monolis_b200_device_clear_matrix": (C.c_int, [_MP]),
    "monolis_b200_device_add_elements_R": (C.c_int, [_MP, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_longlong,
                                                     C.c_void_p]),
    "monolis_b200_device_set_Dirichlet_bc_R": (C.c_int, [_MP, C.c_void_p, C.c_int, _ip, _ip, _dp]),
    "monolis_b200_device_get_values": (C.c_int, [_MP, _dp]),
    "monolis_b200_device_get_diag": (C.c_int, [_MP, _dp]),
    "monolis_b200_nccl_unique_id": (C.c_int, [C.c_void_p]),
    "monolis_b200_com_init_nccl": (C.c_int, [_CP, C.c_void_p, C.c_int, C.c_int]),
    "monolis_b200_com_finalize_nccl": (None, [_CP]),
    "monolis_b200_device_solve_multi_R": (C.c_int, [_MP, C.c_int, C.c_void_p, C.c_void_p, _ip, _dp, _ip]),
}

_ORACLE_EXTRA = {
    "oracle_set_threads": (None, [C.c_int]),
    "oracle_get_threads": (C.c_int, []),
    "oracle_set_iter_rr": (None, [C.c_int]),
    "oracle_set_iter_clock": (None, [_dp, C.c_int]),
    "oracle_pattern_by_simple_mesh_flat": (None, [_MP, C.c_int, C.c_int, C.c_int, C.c_int, _ip]),
    "oracle_add_elements": (None, [_MP, C.c_int, C.c_int, _ip, _dp, C.c_longlong, _dp]),
    "oracle_diag_setup": (None, [_MP, _dp]),
    "oracle_diag_apply": (None, [_MP, _dp, _dp, _dp]),
    "oracle_dot": (C.c_double, [C.c_longlong, _dp, _dp]),
    "oracle_sorted_dot": (C.c_double, [C.c_longlong, _dp, _dp]),
    "oracle_dot_n128": (C.c_double, [C.c_longlong, _dp, _dp]),
    "oracle_set_dot_mode": (None, [C.c_int]),
    "oracle_get_dot_mode": (C.c_int, []),
    "oracle_check_converge": (C.c_int, [_MP, C.c_longlong, _dp, C.c_double, C.c_int]),
}

PRODUCT_SYMBOLS = sorted(list(_COMMON) + list(_PRODUCT))


class MonolisLib:
    """A loaded library exporting the monolis C API."""

    def __init__(self, path: str, extra: dict | None = None):
        if not os.path.exists(path):
            raise FileNotFoundError(f"monolis library not found: {path} (build it with __graft_entry__.build())")
        self.path = path
        self.dll = C.CDLL(path, mode=C.RTLD_LOCAL)
        self.is_product = hasattr(self.dll, "monolis_b200_stream")
        table = dict(_COMMON)
        table.update(_PRODUCT if self.is_product else {})
        if extra:
            table.update(extra)
        for name, (res, args) in table.items():
            fn = getattr(self.dll, name)
            fn.restype = res
            fn.argtypes = args
            setattr(self, name, fn)


def load_product() -> MonolisLib:
    return MonolisLib(PRODUCT_SO)


def load_library(path: str, oracle: bool = False) -> MonolisLib:
    return MonolisLib(path, _ORACLE_EXTRA if oracle else None)


def _iptr(a):
    return a.ctypes.data_as(_ip)


def _dptr(a):
    return a.ctypes.data_as(_dp)


class Monolis:
    """One MONOLIS struct bound to a library; reference-named methods."""

    def __init__(self, lib: MonolisLib):
        self.lib = lib
        self.s = MONOLIS()
        self.p = C.pointer(self.s)
        lib.monolis_initialize(self.p)
        self.com = MONOLIS_COM()
        lib.monolis_com_initialize_by_self(C.pointer(self.com))
        self._alive = True

    def finalize(self):
        if self._alive:
            if getattr(self, "_halo", None) is not None:
                if self.lib.is_product:
                    self.lib.monolis_b200_com_finalize_nccl(C.pointer(self.com))
                self._restore_com()
            self.lib.monolis_finalize(self.p)
            self.lib.monolis_com_finalize(C.pointer(self.com))
            self._alive = False

    # ---- multi-rank tables (product) ----
    def set_halo(self, part, rank, size):
        """Point this struct's MONOLIS_COM at the halo tables of a rank-local
        system (monolis_b200.partition.partition_rows); the arrays stay owned
        by Python and are detached again before the struct is finalized."""
        c = self.com
        self._halo_saved = (c.recv_index, c.send_index)
        keep = {k: np.ascontiguousarray(part[k], dtype=np.int32)
                for k in ("recv_pe", "recv_index", "recv_item", "send_pe", "send_index", "send_item")}
        self._halo = keep
        c.my_rank, c.comm_size, c.n_internal_vertex = rank, size, int(part["N"])
        c.recv_n_neib, c.send_n_neib = len(keep["recv_pe"]), len(keep["send_pe"])
        c.recv_neib_pe, c.recv_index, c.recv_item = (_iptr(keep["recv_pe"]), _iptr(keep["recv_index"]),
                                                     _iptr(keep["recv_item"]))
        c.send_neib_pe, c.send_index, c.send_item = (_iptr(keep["send_pe"]), _iptr(keep["send_index"]),
                                                     _iptr(keep["send_item"]))

    def _restore_com(self):
        c = self.com
        c.recv_index, c.send_index = self._halo_saved
        c.recv_neib_pe = c.recv_item = c.send_neib_pe = c.send_item = None
        c.recv_n_neib = c.send_n_neib = 0
        self._halo = None

    def com_init_nccl(self, uid: bytes, rank, size):
        buf = C.create_string_buffer(bytes(uid), 128)
        rc = self.lib.monolis_b200_com_init_nccl(C.pointer(self.com), buf, rank, size)
        if rc:
            raise RuntimeError(f"com_init_nccl failed: {STATUS_NAMES.get(rc, rc)}")

    def __del__(self):
        try:
            self.finalize()
        except Exception:
            pass

    # ---- parameters ----
    @property
    def Iarray(self):
        return self.s.prm.Iarray

    @property
    def Rarray(self):
        return self.s.prm.Rarray

    def set_method(self, m):
        self.lib.monolis_set_method(self.p, m)

    def set_precond(self, p):
        self.lib.monolis_set_precond(self.p, p)

    def set_maxiter(self, n):
        self.lib.monolis_set_maxiter(self.p, n)

    def set_tolerance(self, t):
        self.lib.monolis_set_tolerance(self.p, t)

    def set_init_x(self, b):
        self.lib.monolis_set_init_x(self.p, bool(b))

    def set_error_abort(self, b):
        self.lib.monolis_set_error_abort(self.p, bool(b))

    def show_iterlog(self, b):
        self.lib.monolis_show_iterlog(self.p, bool(b))

    def show_timelog(self, b):
        self.lib.monolis_show_timelog(self.p, bool(b))

    def show_summary(self, b):
        self.lib.monolis_show_summary(self.p, bool(b))

    def quiet(self):
        self.show_iterlog(False)
        self.show_timelog(False)
        self.show_summary(False)

    def set_precision(self, p):
        rc = self.lib.monolis_b200_set_precision(self.p, p)
        if rc:
            raise ValueError(f"bad precision {p}")

    def matrix_changed(self):
        """monolis_b200_matrix_changed: the host arrays were written directly."""
        self.lib.monolis_b200_matrix_changed(self.p)

    def set_matrix_cache(self, b):
        self.lib.monolis_b200_set_matrix_cache(self.p, bool(b))

    def get_converge_iter(self):
        v = C.c_int()
        self.lib.monolis_get_converge_iter(self.p, C.byref(v))
        return v.value

    def get_converge_residual(self):
        v = C.c_double()
        self.lib.monolis_get_converge_residual(self.p, C.byref(v))
        return v.value

    def get_error_tag(self):
        v = C.c_int()
        self.lib.monolis_get_error_tag(self.p, C.byref(v))
        return v.value

    # ---- pattern / assembly ----
    def get_nonzero_pattern_by_simple_mesh(self, n_node, n_base, n_dof, elem):
        elem = np.ascontiguousarray(elem, dtype=np.int32).reshape(-1, n_base)
        rows = (_ip * len(elem))(*[_iptr(elem[e]) for e in range(len(elem))])
        self.lib.monolis_get_nonzero_pattern_by_simple_mesh_R(self.p, n_node, n_base, n_dof, len(elem), rows)

    def get_nonzero_pattern_flat(self, n_node, n_base, n_dof, elem):
        """Bulk twin of get_nonzero_pattern_by_simple_mesh (flat int32 elem)."""
        elem = np.ascontiguousarray(elem, dtype=np.int32).reshape(-1)
        n_elem = len(elem) // n_base
        if self.lib.is_product:
            rc = self.lib.monolis_b200_get_nonzero_pattern_by_simple_mesh_flat_R(self.p, n_node, n_base, n_dof,
                                                                                 n_elem, _iptr(elem))
            if rc:
                raise ValueError("bad mesh")
        else:
            self.lib.oracle_pattern_by_simple_mesh_flat(self.p, n_node, n_base, n_dof, n_elem, _iptr(elem))

    def get_nonzero_pattern_by_nodal_graph(self, n_node, n_dof, index, item):
        index = np.ascontiguousarray(index, dtype=np.int32)
        item = np.ascontiguousarray(item, dtype=np.int32)
        self.lib.monolis_get_nonzero_pattern_by_nodal_graph_R(self.p, n_node, n_dof, _iptr(index), _iptr(item))

    def add_scalar(self, i, j, si, sj, val):
        self.lib.monolis_add_scalar_to_sparse_matrix_R(self.p, i, j, si, sj, float(val))

    def set_scalar(self, i, j, si, sj, val):
        self.lib.monolis_set_scalar_to_sparse_matrix_R(self.p, i, j, si, sj, float(val))

    def get_scalar(self, i, j, si, sj):
        v = C.c_double()
        f = C.c_bool()
        self.lib.monolis_get_scalar_from_sparse_matrix_R(self.p, i, j, si, sj, C.byref(v), C.byref(f))
        return v.value, f.value

    def add_matrix(self, conn, val):
        conn = np.ascontiguousarray(conn, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        rows = (_dp * val.shape[0])(*[_dptr(val[i]) for i in range(val.shape[0])])
        self.lib.monolis_add_matrix_to_sparse_matrix_R(self.p, len(conn), _iptr(conn), rows)

    def add_elements(self, elem, n_base, val, val_stride, scale=None):
        """Element-by-element add_matrix (bulk entry point of each library)."""
        elem = np.ascontiguousarray(elem, dtype=np.int32).reshape(-1)
        val = np.ascontiguousarray(val, dtype=np.float64)
        n_elem = len(elem) // n_base
        sp = _dptr(np.ascontiguousarray(scale, dtype=np.float64)) if scale is not None else None
        if scale is not None:
            scale = np.ascontiguousarray(scale, dtype=np.float64)
            sp = _dptr(scale)
        if self.lib.is_product:
            rc = self.lib.monolis_b200_add_elements_R(self.p, n_elem, n_base, _iptr(elem), _dptr(val), val_stride, sp)
            if rc:
                raise ValueError("add_elements failed")
        else:
            self.lib.oracle_add_elements(self.p, n_elem, n_base, _iptr(elem), _dptr(val), val_stride, sp)

    def set_matrix_BCSR(self, n, np_, n_dof, nz, A, index, item):
        A = np.ascontiguousarray(A, dtype=np.float64)
        index = np.ascontiguousarray(index, dtype=np.int32)
        item = np.ascontiguousarray(item, dtype=np.int32)
        self.lib.monolis_set_matrix_BCSR_R(self.p, n, np_, n_dof, nz, _dptr(A), _iptr(index), _iptr(item))

    def set_Dirichlet_bc(self, b, node_id, n_dof_bc, val):
        assert b.dtype == np.float64 and b.flags.c_contiguous
        self.lib.monolis_set_Dirichlet_bc_R(self.p, _dptr(b), int(node_id), int(n_dof_bc), float(val))

    # ---- array views of the struct (shared memory, not copies) ----
    @property
    def N(self):
        return self.s.mat.N

    @property
    def NDOF(self):
        return self.s.mat.NDOF

    @property
    def NZ(self):
        return int(self.csr_index()[-1])

    def csr_index(self):
        return np.ctypeslib.as_array(self.s.mat.CSR.index, shape=(self.s.mat.NP + 1,))

    def csr_item(self):
        return np.ctypeslib.as_array(self.s.mat.CSR.item, shape=(int(self.csr_index()[-1]),))

    def csc_index(self):
        return np.ctypeslib.as_array(self.s.mat.CSC.index, shape=(self.s.mat.NP + 1,))

    def csc_item(self):
        return np.ctypeslib.as_array(self.s.mat.CSC.item, shape=(int(self.csr_index()[-1]),))

    def csc_perm(self):
        return np.ctypeslib.as_array(self.s.mat.CSC.perm, shape=(int(self.csr_index()[-1]),))

    def values(self):
        nd = self.s.mat.NDOF
        return np.ctypeslib.as_array(self.s.mat.R.A, shape=(int(self.csr_index()[-1]) * nd * nd,))

    # ---- linear algebra / solve ----
    def matvec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        self.lib.monolis_matvec_product_R(self.p, C.pointer(self.com), _dptr(x), _dptr(y))
        return y

    def inner_product(self, n_dof, x, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        s = C.c_double()
        self.lib.monolis_inner_product_R(self.p, C.pointer(self.com), n_dof, _dptr(x), _dptr(y), C.byref(s))
        return s.value

    def solve(self, b, x):
        """monolis_solve_R(mat, com, b, x): x is updated in place."""
        assert b.dtype == np.float64 and x.dtype == np.float64 and x.flags.c_contiguous
        b = np.ascontiguousarray(b)
        self.lib.monolis_solve_R(self.p, C.pointer(self.com), _dptr(b), _dptr(x))
        return x

    # ---- adjoint pieces (product only) ----
    def solve_transpose(self, b, x):
        """monolis_b200_solve_transpose_R: A^T x = b, x updated in place."""
        assert b.dtype == np.float64 and x.dtype == np.float64 and x.flags.c_contiguous
        b = np.ascontiguousarray(b)
        return self.lib.monolis_b200_solve_transpose_R(self.p, C.pointer(self.com), _dptr(b), _dptr(x))

    def matvec_transpose(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        rc = self.lib.monolis_b200_matvec_transpose_R(self.p, C.pointer(self.com), _dptr(x), _dptr(y))
        if rc:
            raise RuntimeError(f"matvec_transpose failed: {STATUS_NAMES.get(rc, rc)}")
        return y

    def sampled_outer_product(self, lam, x, scale=-1.0):
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        nd = self.NDOF
        G = np.empty(self.NZ * nd * nd)
        rc = self.lib.monolis_b200_sampled_outer_product_R(self.p, _dptr(lam), _dptr(x), scale, _dptr(G))
        if rc:
            raise RuntimeError(f"sampled_outer_product failed: {STATUS_NAMES.get(rc, rc)}")
        return G

    def element_gradient(self, elem, n_base, Ke, ke_stride, lam, x, fixed=None, scale=-1.0):
        elem = np.ascontiguousarray(elem, dtype=np.int32)
        Ke = np.ascontiguousarray(Ke, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        n_elem = elem.size // n_base
        grad = np.empty(n_elem)
        fx = None if fixed is None else np.ascontiguousarray(fixed, dtype=np.int32)
        rc = self.lib.monolis_b200_element_gradient_R(self.p, n_elem, n_base, _iptr(elem), _dptr(Ke), ke_stride,
                                                      _dptr(lam), _dptr(x), None if fx is None else _iptr(fx),
                                                      scale, _dptr(grad))
        if rc:
            raise RuntimeError(f"element_gradient failed: {STATUS_NAMES.get(rc, rc)}")
        return grad

    def solve_multi(self, B):
        """monolis_b200_solve_multi_R: B is (n_rhs, N*ndof); returns (X, iter, resid, status)."""
        B = np.ascontiguousarray(B, dtype=np.float64)
        nr = B.shape[0]
        X = np.zeros_like(B)
        it = np.zeros(nr, dtype=np.int32)
        res = np.zeros(nr)
        st = np.zeros(nr, dtype=np.int32)
        rc = self.lib.monolis_b200_solve_multi_R(self.p, C.pointer(self.com), nr, _dptr(B), _dptr(X), _iptr(it),
                                                 _dptr(res), _iptr(st))
        if rc:
            raise RuntimeError(f"solve_multi failed: {STATUS_NAMES.get(rc, rc)}")
        return X, it, res, st

    # ---- device entry points (product only) ----
    def device_prepare(self):
        rc = self.lib.monolis_b200_device_prepare(self.p)
        if rc:
            raise RuntimeError(f"device_prepare failed: {STATUS_NAMES.get(rc, rc)}")

    def device_solve(self, d_b_ptr, d_x_ptr):
        return self.lib.monolis_b200_device_solve_R(self.p, C.c_void_p(d_b_ptr), C.c_void_p(d_x_ptr))

    def device_solve_com(self, d_b_ptr, d_x_ptr):
        """monolis_b200_device_solve_com_R with this struct's MONOLIS_COM."""
        return self.lib.monolis_b200_device_solve_com_R(self.p, C.pointer(self.com), C.c_void_p(d_b_ptr),
                                                        C.c_void_p(d_x_ptr))

    def device_matvec(self, d_x_ptr, d_y_ptr, fp32=False):
        fn = self.lib.monolis_b200_device_matvec_R32 if fp32 else self.lib.monolis_b200_device_matvec_R
        rc = fn(self.p, C.c_void_p(d_x_ptr), C.c_void_p(d_y_ptr))
        if rc:
            raise RuntimeError(f"device_matvec failed: {STATUS_NAMES.get(rc, rc)}")

    def device_info(self):
        nz = C.c_longlong()
        pad = C.c_longlong()
        ns = C.c_int()
        rc = self.lib.monolis_b200_device_info(self.p, C.byref(nz), C.byref(pad), C.byref(ns))
        if rc:
            raise RuntimeError("device_info: matrix not prepared")
        return nz.value, pad.value, ns.value


class Batch:
    """monolis_b200_batch_*: independent systems solved together by CG in one
    persistent kernel."""

    def __init__(self, lib: MonolisLib):
        self.lib = lib
        self.h = C.c_void_p()
        _check(lib.monolis_b200_batch_create(C.byref(self.h)), "batch_create")
        self.sizes = []
        self.ndof = None

    def add_system(self, m: "Monolis"):
        _check(self.lib.monolis_b200_batch_add_system(self.h, m.p), "batch_add_system")
        self.sizes.append(m.N * m.NDOF)
        self.ndof = m.NDOF

    def add_csr(self, n, ndof, index, item, val):
        index = np.ascontiguousarray(index, dtype=np.int32)
        item = np.ascontiguousarray(item, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        _check(self.lib.monolis_b200_batch_add_csr(self.h, n, ndof, _iptr(index), _iptr(item), _dptr(val)),
               "batch_add_csr")
        self.sizes.append(n * ndof)
        self.ndof = ndof

    def prepare(self, precond=1, autotune=True):
        _check(self.lib.monolis_b200_batch_prepare(self.h, precond, int(autotune)), "batch_prepare")

    def set_config(self, cluster, threads, split_rows):
        _check(self.lib.monolis_b200_batch_set_config(self.h, cluster, threads, split_rows), "batch_set_config")

    def config(self):
        c, t, sp = C.c_int(), C.c_int(), C.c_longlong()
        _check(self.lib.monolis_b200_batch_get_config(self.h, C.byref(c), C.byref(t), C.byref(sp)), "batch_config")
        return c.value, t.value, sp.value

    def unroll(self):
        u = C.c_int()
        _check(self.lib.monolis_b200_batch_get_unroll(self.h, C.byref(u)), "batch_unroll")
        return u.value

    def autotune(self, iters=30, cap=64):
        n = C.c_int(cap)
        cl = (C.c_int * cap)()
        th = (C.c_int * cap)()
        sp = (C.c_longlong * cap)()
        sec = (C.c_double * cap)()
        _check(self.lib.monolis_b200_batch_autotune(self.h, iters, C.byref(n), cl, th, sp, sec), "batch_autotune")
        return [(cl[i], th[i], sp[i], sec[i]) for i in range(min(n.value, cap))]

    def solve(self, bs, tol=1e-8, max_iter=10000, refine=True):
        """Host right-hand sides (list of arrays) -> (xs, iters, resid, status)."""
        ns = len(self.sizes)
        bs = [np.ascontiguousarray(b, dtype=np.float64) for b in bs]
        xs = [np.zeros(n) for n in self.sizes]
        bp = (_dp * ns)(*[_dptr(b) for b in bs])
        xp = (_dp * ns)(*[_dptr(x) for x in xs])
        it = np.zeros(ns, dtype=np.int32)
        res = np.zeros(ns)
        st = np.zeros(ns, dtype=np.int32)
        _check(self.lib.monolis_b200_batch_solve_R(self.h, bp, xp, tol, max_iter, int(refine), _iptr(it), _dptr(res),
                                                   _iptr(st)), "batch_solve")
        return xs, it, res, st

    def offsets(self):
        n = C.c_int()
        _check(self.lib.monolis_b200_batch_info(self.h, C.byref(n), None), "batch_info")
        off = (C.c_longlong * n.value)()
        _check(self.lib.monolis_b200_batch_info(self.h, C.byref(n), off), "batch_info")
        return np.array(off[:], dtype=np.int64)

    def device_vectors(self):
        db, dx = C.c_void_p(), C.c_void_p()
        _check(self.lib.monolis_b200_batch_device_vectors(self.h, C.byref(db), C.byref(dx)), "batch_device_vectors")
        return db.value, dx.value

    def device_solve(self, tol=1e-8, max_iter=10000, refine=True):
        ns = len(self.sizes)
        it = np.zeros(ns, dtype=np.int32)
        res = np.zeros(ns)
        st = np.zeros(ns, dtype=np.int32)
        _check(self.lib.monolis_b200_batch_device_solve_R(self.h, tol, max_iter, int(refine), _iptr(it), _dptr(res),
                                                          _iptr(st)), "batch_device_solve")
        return it, res, st

    def last_seconds(self):
        return self.lib.monolis_b200_batch_last_seconds(self.h)

    def destroy(self):
        if self.h:
            self.lib.monolis_b200_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def _check(rc, what):
    if rc:
        raise RuntimeError(f"{what} failed: {STATUS_NAMES.get(rc, rc)}")


def nccl_unique_id(lib: MonolisLib) -> bytes:
    """An NCCL unique id (128 bytes) for monolis_b200_com_init_nccl."""
    buf = C.create_string_buffer(128)
    rc = lib.monolis_b200_nccl_unique_id(buf)
    if rc:
        raise RuntimeError(f"nccl_unique_id failed: {STATUS_NAMES.get(rc, rc)}")
    return buf.raw


def stream_handle(lib: MonolisLib) -> int:
    """cudaStream_t of the library (all its device work runs there)."""
    return lib.monolis_b200_stream() or 0
