"""ctypes binding of librgpu.so (the C ABI declared in include/rgpu.h).

This is the Python face of the same extern "C" boundary a C++ host (the
GpuHydroSolver patch) calls; tests and bench.py use it.  It loads the
in-tree library and fails loudly when it is missing: there is no CPU
fallback on this path.
"""
import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "librgpu.so"

I32P = C.POINTER(C.c_int)
F64P = C.POINTER(C.c_double)

RG_OK, RG_ERR_ARG, RG_ERR_CUDA, RG_ERR_UNSUPPORTED, RG_ERR_TOPOLOGY, RG_ERR_STATE, RG_ERR_TIMEOUT, RG_ERR_DEVICE, \
    RG_ERR_NOMEM = 0, -1, -2, -3, -4, -5, -6, -7, -8
RIEMANN = {"llf": 0, "hll": 1, "hllc": 2, "exact": 3, "acoustic": 4}


class rg_params(C.Structure):
    _fields_ = [("ndim", C.c_int), ("nvar", C.c_int), ("slope_type", C.c_int), ("riemann", C.c_int),
                ("interpol_type", C.c_int), ("interpol_var", C.c_int), ("gamma", C.c_double),
                ("courant_factor", C.c_double), ("exact_niter", C.c_int), ("exact_tol", C.c_double),
                ("exact_guess", C.c_int), ("boxlen", C.c_double), ("flags", C.c_int)]


class rg_grid_view(C.Structure):
    _fields_ = [("ncoarse", C.c_int), ("ngridmax", C.c_int), ("ncell", C.c_int), ("nvar", C.c_int),
                ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("ncpu", C.c_int),
                ("nboundary", C.c_int), ("nlevelmax", C.c_int),
                ("son", I32P), ("father", I32P), ("nbor", I32P), ("next", I32P), ("headl", I32P),
                ("bound_type", I32P), ("nbound_type", C.c_int)]


class rg_tree_arrays(C.Structure):
    _fields_ = [(k, I32P) for k in ("son", "father", "nbor", "next", "prev", "headl", "taill", "numbl", "flag1",
                                    "flag2", "cpu_map")] + \
               [("xg", C.POINTER(C.c_double)), ("uold", C.POINTER(C.c_double)), ("unew", C.POINTER(C.c_double)),
                ("headf", C.c_int), ("tailf", C.c_int), ("numbf", C.c_int)]


class rg_amr_config(C.Structure):
    _fields_ = [("levelmin", C.c_int), ("nexpand", C.c_int), ("courant_factor", C.c_double),
                ("err_grad_d", C.c_double), ("err_grad_p", C.c_double), ("err_grad_u", C.c_double),
                ("pressure_cap", C.c_int), ("boxlen", C.c_double)]


class rg_amr_clock(C.Structure):
    _fields_ = [("dtnew", C.c_double * 33), ("dtold", C.c_double * 33), ("t", C.c_double), ("nstep", C.c_int64),
                ("cell_updates", C.c_int64)]


class rg_plan_info(C.Structure):
    _fields_ = [(k, C.c_int) for k in ("ncells", "ntarg", "nevents", "nextra_prim", "nlong")]


TREE_INT_ARRAYS = ("son", "father", "nbor", "next", "prev", "headl", "taill", "numbl", "flag1", "flag2", "cpu_map")
TREE_F64_ARRAYS = ("xg", "uold", "unew")


def tree_arrays(d):
    """rg_tree_arrays over a dict of contiguous numpy arrays (int32 / float64)
    and the scalars headf, tailf, numbf; the arrays are written in place by
    rg_tree_fetch."""
    t = rg_tree_arrays()
    for k in TREE_INT_ARRAYS:
        a = d[k]
        assert a.dtype == np.int32 and a.flags.c_contiguous
        setattr(t, k, a.ctypes.data_as(I32P))
    for k in TREE_F64_ARRAYS:
        a = d[k]
        assert a.dtype == np.float64 and a.flags.c_contiguous
        setattr(t, k, a.ctypes.data_as(C.POINTER(C.c_double)))
    t.headf, t.tailf, t.numbf = int(d["headf"]), int(d["tailf"]), int(d["numbf"])
    t._keep = d
    return t


def make_params(ndim, nvar=None, slope_type=1, riemann="hllc", interpol_type=1, interpol_var=0, gamma=1.4,
                courant_factor=0.8, exact_niter=10, exact_tol=1e-6, exact_guess=0, boxlen=1.0):
    r = RIEMANN.get(riemann, 0) if isinstance(riemann, str) else int(riemann)
    return rg_params(ndim, nvar if nvar else ndim + 2, slope_type, r, interpol_type, interpol_var, gamma,
                     courant_factor, exact_niter, exact_tol, exact_guess, boxlen, 0)


def grid_view(g):
    """rg_grid_view over an object with the AmrGrid scalars and int32 arrays."""
    v = rg_grid_view()
    for k in ("ncoarse", "ngridmax", "ncell", "nvar", "nx", "ny", "nz", "ncpu", "nboundary", "nlevelmax"):
        setattr(v, k, int(getattr(g, k)))
    keep = []
    for k in ("son", "father", "nbor", "next", "headl"):
        a = np.ascontiguousarray(getattr(g, k), dtype=np.int32)
        keep.append(a)
        setattr(v, k, a.ctypes.data_as(I32P))
    v.bound_type = None
    v.nbound_type = 0
    v._keep = keep
    return v


_lib = None


def lib():
    """Load librgpu.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run ramses-cpp_b200/build.py (no CPU fallback exists)")
    L = C.CDLL(str(LIB_PATH))
    P = C.POINTER(rg_params)
    L.rg_create.restype = C.c_void_p
    L.rg_create.argtypes = [P, C.c_int]
    L.rg_destroy.argtypes = [C.c_void_p]
    L.rg_last_error.restype = C.c_char_p
    L.rg_last_error.argtypes = [C.c_void_p]
    L.rg_version.restype = C.c_char_p
    L.rg_riemann_from_string.argtypes = [C.c_char_p]
    L.rg_set_params.argtypes = [C.c_void_p, P]
    L.rg_sync_topology.argtypes = [C.c_void_p, C.POINTER(rg_grid_view)]
    L.rg_upload_state.argtypes = [C.c_void_p, F64P, F64P]
    L.rg_download_state.argtypes = [C.c_void_p, F64P, F64P]
    L.rg_device_state.argtypes = [C.c_void_p, C.POINTER(F64P), C.POINTER(F64P)]
    L.rg_set_unew.argtypes = [C.c_void_p, C.c_int]
    L.rg_set_uold.argtypes = [C.c_void_p, C.c_int]
    L.rg_godunov_level.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
    L.rg_courant_step.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int, F64P]
    L.rg_level_substep.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, F64P]
    L.rg_synchronize.argtypes = [C.c_void_p]
    L.rg_level_octs.argtypes = [C.c_void_p, C.c_int, I32P, C.c_int, I32P]
    L.rg_level_nbor_cells.argtypes = [C.c_void_p, C.c_int, I32P, C.c_int]
    L.rg_level_cell_updates.restype = C.c_int64
    L.rg_level_cell_updates.argtypes = [C.c_void_p, C.c_int]
    L.rg_last_kernel_ms.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_int]
    L.rg_pool_usage.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.rg_kernel_ms_totals.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int64), C.c_int]
    L.rg_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.rg_set_timing.argtypes = [C.c_void_p, C.c_int]
    L.rg_exact_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_int]
    L.rg_set_autotune.argtypes = [C.c_void_p, C.c_int]
    L.rg_set_face_config.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
    VP = C.c_void_p
    L.rg_exact_batch.argtypes = [VP, C.c_int, VP, VP, VP, VP, VP, VP, C.c_int, C.c_int, C.c_double]
    L.rg_stress_states.argtypes = [VP, C.c_int, C.c_uint64, VP, VP, VP]
    L.rg_mlp_train.argtypes = [VP, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint64, C.POINTER(C.c_float)]
    L.rg_mlp_get.argtypes = [VP, C.POINTER(C.c_float)]
    L.rg_mlp_set.argtypes = [VP, C.POINTER(C.c_float)]
    L.rg_mlp_grad.argtypes = [VP, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                              C.POINTER(C.c_float)]
    L.rg_face_config.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float)]
    L.rg_godunov_level_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    L.rg_get_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    L.rg_godunov_level_host.argtypes = [VP, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double)]
    L.rg_set_level_boxes.argtypes = [VP, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.rg_level_box_dt.argtypes = [VP, C.c_int, C.POINTER(C.c_double), C.c_int]
    IP = C.POINTER(C.c_int)
    L.rg_set_level_lattices.argtypes = [VP, C.c_int, C.c_int, IP, IP, IP]
    L.rg_level_output.argtypes = [VP, C.c_int, C.POINTER(C.c_double), C.c_int64]
    L.rg_level_substep_host.argtypes = [VP, C.c_int, C.c_double, C.c_int, VP, VP, C.POINTER(C.c_double)]
    TP = C.POINTER(rg_tree_arrays)
    L.rg_tree_attach.argtypes = [VP, C.POINTER(rg_grid_view), TP, C.c_int]
    L.rg_tree_fetch.argtypes = [VP, TP]
    L.rg_flag_fine.argtypes = [VP, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]
    L.rg_make_grid_fine.argtypes = [VP, C.c_int]
    L.rg_remove_grid_fine.argtypes = [VP, C.c_int]
    L.rg_restrict_fine.argtypes = [VP, C.c_int]
    L.rg_count_grids.argtypes = [VP, C.c_int, IP]
    L.rg_tree_sizes.argtypes = [VP, IP, IP]
    L.rg_level_plan_info.argtypes = [VP, C.c_int, C.POINTER(rg_plan_info)]
    L.rg_amr_coarse_step.argtypes = [VP, C.POINTER(rg_amr_config), C.POINTER(rg_amr_clock)]
    L.rg_amr_graphs.argtypes = [VP, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.rg_measure_fp64_peak.argtypes = [VP, C.POINTER(C.c_double)]
    L.rg_level_run.argtypes = [VP, C.c_int, C.c_double, C.c_int, C.c_double, C.c_double, C.c_int64,
                               C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    _lib = L
    return L


class RGError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rgpu error {code}: {msg}")
        self.code = code


def _f64(a):
    return a.ctypes.data_as(F64P) if a is not None else None


class Context:
    """One rg_ctx: device mirror of an AmrGrid plus the level-step kernels."""

    def __init__(self, params, device=-1):
        self.L = lib()
        self.params = params
        self.h = self.L.rg_create(C.byref(params), device)
        if not self.h:
            raise RGError(RG_ERR_NOMEM, "rg_create returned NULL")
        self._view = None
        self.ncell = 0
        self.nvar = params.nvar

    def _chk(self, rc):
        if rc != RG_OK:
            raise RGError(rc, self.L.rg_last_error(self.h).decode())
        return rc

    def close(self):
        if self.h:
            self.L.rg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params):
        self.params = params
        self._chk(self.L.rg_set_params(self.h, C.byref(params)))

    def sync_topology(self, g):
        self._view = grid_view(g)
        self.ncell = int(g.ncell)
        self._chk(self.L.rg_sync_topology(self.h, C.byref(self._view)))

    # -- device-resident tree (TreeUpdater on the GPU) ---------------------------
    def tree_attach(self, g, arrays, levelmin):
        """Take over the tree: g gives sizes and son/father/nbor/next/headl,
        arrays (a dict like RefHarness.tree_arrays) the rest and the state."""
        self._view = grid_view(g)
        self.ncell = int(g.ncell)
        d = {k: np.ascontiguousarray(arrays[k], dtype=np.int32) for k in TREE_INT_ARRAYS}
        d.update({k: np.ascontiguousarray(arrays[k], dtype=np.float64) for k in TREE_F64_ARRAYS})
        d.update(headf=arrays["headf"], tailf=arrays["tailf"], numbf=arrays["numbf"])
        self._tree = tree_arrays(d)
        self._chk(self.L.rg_tree_attach(self.h, C.byref(self._view), C.byref(self._tree), int(levelmin)))

    def tree_sizes(self):
        """(ngridmax, ncell) of the context's tree: both grow when make_grid_fine runs out of free octs."""
        g, n = C.c_int(0), C.c_int(0)
        self._chk(self.L.rg_tree_sizes(self.h, C.byref(g), C.byref(n)))
        return g.value, n.value

    def tree_fetch(self, like):
        """Fresh numpy copies of every tree array and the state, sized by the
        device tree (the level-list arrays by `like`)."""
        ngm, ncell = self.tree_sizes()
        nv = self.nvar
        per = {"son": ncell, "father": ngm, "nbor": 6 * ngm, "next": ngm, "prev": ngm, "flag1": ncell,
               "flag2": ncell, "cpu_map": ncell, "xg": 3 * ngm, "uold": nv * ncell, "unew": nv * ncell}
        d = {k: np.zeros(per[k] if k in per else len(like[k]), dtype=np.int32) for k in TREE_INT_ARRAYS}
        d.update({k: np.zeros(per[k], dtype=np.float64) for k in TREE_F64_ARRAYS})
        d.update(headf=0, tailf=0, numbf=0)
        t = tree_arrays(d)
        self._chk(self.L.rg_tree_fetch(self.h, C.byref(t)))
        d.update(headf=t.headf, tailf=t.tailf, numbf=t.numbf)
        return d

    def flag_fine(self, il, ed=-1.0, ep=-1.0, ev=-1.0, eb2=-1.0, nexp=1, icount=1, nsub=2):
        self._chk(self.L.rg_flag_fine(self.h, il, ed, ep, ev, eb2, nexp, icount, nsub))

    def make_grid_fine(self, il):
        self._chk(self.L.rg_make_grid_fine(self.h, il))

    def remove_grid_fine(self, il):
        self._chk(self.L.rg_remove_grid_fine(self.h, il))

    def restrict_fine(self, il):
        self._chk(self.L.rg_restrict_fine(self.h, il))

    def amr_coarse_step(self, cfg, clock):
        """rg_amr_coarse_step: one coarse step of the resident run (clock updated in place)."""
        self._chk(self.L.rg_amr_coarse_step(self.h, C.byref(cfg), C.byref(clock)))

    def amr_graphs(self, on=None):
        """Switch the coarse step's graphs (on=True/False) and return the
        (captured, replayed) counts of runs (the level-step segments between two
        of the host's waits)."""
        cap, rep = C.c_int64(0), C.c_int64(0)
        self._chk(self.L.rg_amr_graphs(self.h, -1 if on is None else (1 if on else 0), C.byref(cap), C.byref(rep)))
        return cap.value, rep.value

    def level_run(self, il, dx, t_end, t_start=0.0, pressure_cap=False, max_steps=10**7):
        """rg_level_run: substeps until t >= t_end in one graph launch; returns (t, steps)."""
        t, n = C.c_double(0), C.c_int64(0)
        self._chk(self.L.rg_level_run(self.h, il, dx, 1 if pressure_cap else 0, t_start, t_end, int(max_steps),
                                      C.byref(t), C.byref(n)))
        return t.value, n.value

    def measure_fp64_peak(self):
        """Device FP64 throughput in TFLOP/s (rg_measure_fp64_peak)."""
        v = C.c_double(0)
        self._chk(self.L.rg_measure_fp64_peak(self.h, C.byref(v)))
        return v.value

    def count_grids(self, il):
        n = C.c_int(0)
        self._chk(self.L.rg_count_grids(self.h, il, C.byref(n)))
        return n.value

    def upload_state(self, uold=None, unew=None):
        self._chk(self.L.rg_upload_state(self.h, _f64(uold), _f64(unew)))

    def download_state(self, uold=None, unew=None):
        self._chk(self.L.rg_download_state(self.h, _f64(uold), _f64(unew)))

    def device_state(self):
        a, b = F64P(), F64P()
        self._chk(self.L.rg_device_state(self.h, C.byref(a), C.byref(b)))
        return C.cast(a, C.c_void_p).value, C.cast(b, C.c_void_p).value

    def set_unew(self, il):
        self._chk(self.L.rg_set_unew(self.h, il))

    def set_uold(self, il):
        self._chk(self.L.rg_set_uold(self.h, il))

    def godunov_level(self, il, dt, dx):
        self._chk(self.L.rg_godunov_level(self.h, il, dt, dx))

    def godunov_level_host(self, il, dt, dx, uold, unew):
        """Level step on host arrays: unew (float64, C-contiguous) is updated in place
        at the step's targets only."""
        if uold.dtype != np.float64 or unew.dtype != np.float64 or not unew.flags.c_contiguous:
            raise ValueError("uold/unew must be contiguous float64 arrays")
        uo = np.ascontiguousarray(uold)
        self._chk(self.L.rg_godunov_level_host(self.h, il, dt, dx, uo.ctypes.data_as(C.POINTER(C.c_double)),
                                               unew.ctypes.data_as(C.POINTER(C.c_double))))

    def level_substep_host_ptr(self, il, dx, uold_ptr, unew_ptr=None, pressure_cap=False, want_dt=True):
        """Substep on host state at raw addresses (e.g. pinned torch tensors): uold is
        read and then updated in place at the level's targets."""
        dt = C.c_double(0)
        self._chk(self.L.rg_level_substep_host(self.h, il, dx, 1 if pressure_cap else 0, uold_ptr, unew_ptr,
                                               C.byref(dt) if want_dt else None))
        return dt.value if want_dt else None

    def godunov_level_noalloc(self, il, dt, dx, uold_dev_ptr, unew_dev_ptr):
        """Allocation-free level step on caller-owned device buffers (raw addresses)."""
        self._chk(self.L.rg_godunov_level_noalloc(self.h, il, dt, dx, C.c_void_p(uold_dev_ptr),
                                                  C.c_void_p(unew_dev_ptr)))

    def courant_step(self, il, dx, cfl, pressure_cap=True):
        out = C.c_double(0)
        self._chk(self.L.rg_courant_step(self.h, il, dx, cfl, 1 if pressure_cap else 0, C.byref(out)))
        return out.value

    def level_substep(self, il, dx, pressure_cap=False, use_graph=True, want_dt=False):
        out = C.c_double(0)
        self._chk(self.L.rg_level_substep(self.h, il, dx, 1 if pressure_cap else 0, 1 if use_graph else 0,
                                          C.byref(out) if want_dt else None))
        return out.value if want_dt else None

    def set_stream(self, stream_handle):
        self._chk(self.L.rg_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None))

    def get_stream(self):
        out = C.c_void_p()
        self._chk(self.L.rg_get_stream(self.h, C.byref(out)))
        return out.value

    def upload_state_ptr(self, uold_ptr=None, unew_ptr=None):
        """Upload from raw host addresses (e.g. pinned torch tensors)."""
        self._chk(self.L.rg_upload_state(self.h, C.cast(C.c_void_p(uold_ptr), F64P) if uold_ptr else None,
                                         C.cast(C.c_void_p(unew_ptr), F64P) if unew_ptr else None))

    def download_state_ptr(self, uold_ptr=None, unew_ptr=None):
        self._chk(self.L.rg_download_state(self.h, C.cast(C.c_void_p(uold_ptr), F64P) if uold_ptr else None,
                                           C.cast(C.c_void_p(unew_ptr), F64P) if unew_ptr else None))

    def synchronize(self):
        self._chk(self.L.rg_synchronize(self.h))

    def plan_info(self, il):
        """rg_level_plan_info as a dict: ncells, ntarg, nevents, nextra_prim, nlong."""
        i = rg_plan_info()
        self._chk(self.L.rg_level_plan_info(self.h, il, C.byref(i)))
        return {k: getattr(i, k) for k, _ in rg_plan_info._fields_}

    def level_octs(self, il):
        n = C.c_int(0)
        self._chk(self.L.rg_level_octs(self.h, il, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1), dtype=np.int32)
        self._chk(self.L.rg_level_octs(self.h, il, out.ctypes.data_as(I32P), n.value, C.byref(n)))
        return out[:n.value]

    def level_nbor_cells(self, il, ncells):
        out = np.zeros(max(ncells * 6, 1), dtype=np.int32)
        self._chk(self.L.rg_level_nbor_cells(self.h, il, out.ctypes.data_as(I32P), out.size))
        return out[:ncells * 6].reshape(ncells, 6)

    def cell_updates(self, il):
        return int(self.L.rg_level_cell_updates(self.h, il))

    def exact_stats(self, reset=False):
        it, ca = C.c_int64(0), C.c_int64(0)
        self._chk(self.L.rg_exact_stats(self.h, C.byref(it), C.byref(ca), 1 if reset else 0))
        return it.value, ca.value

    def set_autotune(self, on):
        self._chk(self.L.rg_set_autotune(self.h, 1 if on else 0))

    def face_config(self, il):
        v, b, ms = C.c_int(0), C.c_int(0), C.c_float(0)
        self._chk(self.L.rg_face_config(self.h, il, C.byref(v), C.byref(b), C.byref(ms)))
        return v.value, b.value, ms.value

    def set_face_config(self, il, variant, batch):
        self._chk(self.L.rg_set_face_config(self.h, il, variant, batch))

    # ---- ensembles of independent boxes sharing one level list
    def set_level_boxes(self, il, first_oct, dx):
        first = np.ascontiguousarray(first_oct, dtype=np.int32)
        dxs = np.ascontiguousarray(dx, dtype=np.float64)
        if len(first) != len(dxs) + 1:
            raise ValueError("first_oct needs one entry more than dx")
        self._chk(self.L.rg_set_level_boxes(self.h, il, len(dxs), first.ctypes.data_as(C.POINTER(C.c_int)),
                                            dxs.ctypes.data_as(C.POINTER(C.c_double))))

    def set_level_lattices(self, il, extent, lat_id, lat_p):
        ext = np.ascontiguousarray(extent, dtype=np.int32).reshape(-1)
        lid = np.ascontiguousarray(lat_id, dtype=np.int32)
        lp = np.ascontiguousarray(lat_p, dtype=np.int32)
        IP = C.POINTER(C.c_int)
        self._chk(self.L.rg_set_level_lattices(self.h, il, len(ext) // 3, ext.ctypes.data_as(IP),
                                               lid.ctypes.data_as(IP), lp.ctypes.data_as(IP)))

    def level_output(self, il, ndim, nvar):
        """Snapshot records of level il: array [2^ndim][nvar][noct] (list order)."""
        noct = len(self.level_octs(il))
        out = np.empty(((1 << ndim), nvar, noct), dtype=np.float64)
        if noct:
            self._chk(self.L.rg_level_output(self.h, il, out.ctypes.data_as(C.POINTER(C.c_double)), out.size))
        return out

    def level_box_dt(self, il, nbox):
        out = np.zeros(nbox, dtype=np.float64)
        self._chk(self.L.rg_level_box_dt(self.h, il, out.ctypes.data_as(C.POINTER(C.c_double)), nbox))
        return out

    # ---- exact solver / learned guess (device buffers passed as raw addresses)
    def exact_batch(self, n, ql, qr, gamma=None, flux=None, pstar=None, iters=None, learned=False, niter=10,
                    tol=1e-6):
        self._chk(self.L.rg_exact_batch(self.h, n, ql, qr, gamma, flux, pstar, iters, 1 if learned else 0, niter,
                                        tol))

    def stress_states(self, n, seed, ql, qr, gamma):
        self._chk(self.L.rg_stress_states(self.h, n, seed, ql, qr, gamma))

    def mlp_train(self, nsamples=10_000_000, epochs=30, batch=8192, lr=2e-3, seed=1):
        loss = C.c_float(0)
        self._chk(self.L.rg_mlp_train(self.h, nsamples, epochs, batch, lr, seed, C.byref(loss)))
        return loss.value

    def mlp_get(self):
        out = np.zeros(self.L.rg_mlp_nparam(), dtype=np.float32)
        self._chk(self.L.rg_mlp_get(self.h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def mlp_set(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._chk(self.L.rg_mlp_set(self.h, p.ctypes.data_as(C.POINTER(C.c_float))))

    def mlp_grad(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(4801, dtype=np.float32)
        loss = C.c_float(0)
        FP = C.POINTER(C.c_float)
        self._chk(self.L.rg_mlp_grad(self.h, len(t), x.ctypes.data_as(FP), t.ctypes.data_as(FP),
                                     g.ctypes.data_as(FP), C.byref(loss)))
        return g, loss.value

    def set_timing(self, on):
        """True/False: events of the last level step; "accumulate": every level step's events."""
        self._chk(self.L.rg_set_timing(self.h, 2 if on == "accumulate" else (1 if on else 0)))

    def kernel_ms_totals(self, reset=True):
        """Accumulated (prim, face, fold) device ms, face-kernel cells and level steps."""
        ms = (C.c_double * 3)()
        cells, steps = C.c_int64(0), C.c_int64(0)
        self._chk(self.L.rg_kernel_ms_totals(self.h, ms, C.byref(cells), C.byref(steps), 1 if reset else 0))
        return list(ms), cells.value, steps.value

    def pool_usage(self):
        """(reserved, used) bytes of the context's device memory pool."""
        r, u = C.c_uint64(0), C.c_uint64(0)
        self._chk(self.L.rg_pool_usage(self.h, C.byref(r), C.byref(u)))
        return r.value, u.value

    def kernel_ms(self):
        out = (C.c_float * 3)()
        rc = self.L.rg_last_kernel_ms(self.h, out, 3)
        return list(out) if rc == RG_OK else None
