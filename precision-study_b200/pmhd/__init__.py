"""Python bindings (ctypes) for libpmhd.so, the B200 2D ideal-MHD + GLM solver.

The C ABI is declared in include/pmhd.h.  This module loads the in-tree
library built by precision-study_b200/Makefile and fails loudly when it is
missing: there is no CPU fallback.

Typical use::

    import pmhd
    with pmhd.Solver(nx=256, ny=256, precision="mixed") as s:
        s.init_problem(pmhd.PROBLEM_ORSZAG_TANG)
        st = s.advance(t_end=0.5)
        U = s.get_state()            # (ny, nx, 9) conserved fields
"""
import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("PMHD_LIB") or os.path.join(PKG_DIR, "libpmhd.so")
CLI_PATH = os.path.join(PKG_DIR, "bin", "mhd2d_glm_gpu")

OK, ERR_ARG, ERR_RATE, ERR_STAGE1, ERR_STAGE2, ERR_IO, ERR_CUDA = 0, 1, 2, 3, 4, 5, 9
ERR_TIMEOUT, ERR_NOMEM, ERR_UNSUPPORTED, ERR_NODEVICE = -1, -2, -3, -4
FP64, FP32, MIXED = 0, 1, 2
BC_PERIODIC, BC_REFLECT, BC_TRANSMISSIVE = 0, 1, 2
ORDER_FIRST, ORDER_MUSCL, ORDER_HANCOCK = 0, 1, 2
SOLVER_HLL, SOLVER_HLLD, SOLVER_HLLC = 0, 1, 2
PROBLEM_ORSZAG_TANG, PROBLEM_KH_REF, PROBLEM_KH_REFLECT, PROBLEM_BRIO_WU_2D, PROBLEM_BRIO_WU_TORUS = 0, 1, 2, 3, 4
LAYOUT_INTERIOR, LAYOUT_GHOSTED = 0, 1
CONV_GELU, CONV_LINEAR, CONV_DGELU = 0, 1, 2

PRECISIONS = {"fp64": FP64, "fp32": FP32, "mixed": MIXED}

# Every entry point include/pmhd.h declares.
EXPORTS = (
    "pmhd_config_default", "pmhd_create", "pmhd_destroy", "pmhd_init_problem",
    "pmhd_set_state", "pmhd_get_state", "pmhd_set_time", "pmhd_advance",
    "pmhd_get_stats", "pmhd_diagnostics", "pmhd_write_dat", "pmhd_dat_filename",
    "pmhd_strerror", "pmhd_get_config", "pmhd_problem_state", "pmhd_advance_noalloc",
    "pmhd_ensemble_describe_default", "pmhd_ensemble_create", "pmhd_ensemble_advance",
    "pmhd_ensemble_member_stats", "pmhd_ensemble_get_state", "pmhd_ensemble_destroy",
    "pmhd_conv3x3", "pmhd_conv3x3_wgrad", "pmhd_learned_loss_grad",
    "pmhd_learned_config_default", "pmhd_learned_create", "pmhd_learned_destroy", "pmhd_learned_generate",
    "pmhd_learned_generate_rollout", "pmhd_learned_generate_corrected",
    "pmhd_learned_num_pairs", "pmhd_learned_train", "pmhd_learned_run", "pmhd_learned_fine_run",
    "pmhd_learned_save", "pmhd_learned_load",
    "pmhd_euler2d_create", "pmhd_euler2d_advance", "pmhd_euler2d_get_prim", "pmhd_euler2d_destroy",
    "pmhd_euler1d_run", "pmhd_write_restart", "pmhd_read_restart",
)


class PmhdError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        super().__init__(f"{where}: {strerror(status)} (status {status})")


class Config(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
        ("y_min", ctypes.c_double), ("y_max", ctypes.c_double),
        ("gamma", ctypes.c_double), ("hlld_tol", ctypes.c_double),
        ("cfl", ctypes.c_double), ("alpha", ctypes.c_double),
        ("order", ctypes.c_int), ("solver", ctypes.c_int),
        ("precision", ctypes.c_int), ("exact", ctypes.c_int),
        ("bc", ctypes.c_int * 4), ("device", ctypes.c_int),
        ("steps_per_graph", ctypes.c_int), ("autotune", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_longlong), ("t", ctypes.c_double),
        ("ch_last", ctypes.c_double), ("dt_last", ctypes.c_double),
        ("x_evals", ctypes.c_ulonglong), ("y_evals", ctypes.c_ulonglong),
        ("degenerate", ctypes.c_ulonglong), ("nonphysical", ctypes.c_ulonglong),
        ("status", ctypes.c_int), ("bad_i", ctypes.c_int), ("bad_j", ctypes.c_int),
        ("bad_step", ctypes.c_longlong), ("kernel_launches", ctypes.c_ulonglong),
        ("device_ms", ctypes.c_double), ("tile_height", ctypes.c_int), ("ctas", ctypes.c_int),
        ("zone_cycles", ctypes.c_ulonglong),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class MemberDesc(ctypes.Structure):
    """pmhd_member_desc: one member of an ensemble."""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
        ("y_min", ctypes.c_double), ("y_max", ctypes.c_double),
        ("gamma", ctypes.c_double), ("bc", ctypes.c_int * 4),
        ("problem", ctypes.c_int), ("nparams", ctypes.c_int), ("params", ctypes.c_double * 4),
        ("t_end", ctypes.c_double),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["bc"] = tuple(self.bc)
        d["params"] = tuple(self.params[:self.nparams])
        return d


class LearnedConfig(ctypes.Structure):
    """pmhd_learned_config."""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("refine", ctypes.c_int),
        ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
        ("y_min", ctypes.c_double), ("y_max", ctypes.c_double),
        ("gamma", ctypes.c_double), ("cfl", ctypes.c_double), ("alpha", ctypes.c_double),
        ("precision", ctypes.c_int), ("device", ctypes.c_int), ("max_pairs", ctypes.c_int),
        ("seed", ctypes.c_ulonglong), ("div_tol", ctypes.c_double), ("relax", ctypes.c_double),
        ("train_noise", ctypes.c_double), ("shrink", ctypes.c_double),
    ]


class LearnedStats(ctypes.Structure):
    """pmhd_learned_stats."""
    _fields_ = [
        ("steps", ctypes.c_longlong), ("t", ctypes.c_double), ("accepted", ctypes.c_longlong),
        ("rejected_positivity", ctypes.c_longlong), ("rejected_divergence", ctypes.c_longlong),
        ("device_ms", ctypes.c_double), ("wall_ms", ctypes.c_double), ("status", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class EulerStats(ctypes.Structure):
    """pmhd_euler_stats."""
    _fields_ = [("steps", ctypes.c_longlong), ("t", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("status", ctypes.c_int)]


_lib = None


def load():
    """Load libpmhd.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}`")
    L = ctypes.CDLL(LIB_PATH)
    P, vp, i, d = ctypes.POINTER, ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    sig = {
        "pmhd_config_default": ([P(Config)], i),
        "pmhd_create": ([P(Config), P(vp)], i),
        "pmhd_destroy": ([vp], i),
        "pmhd_init_problem": ([vp, i, P(d), i], i),
        "pmhd_set_state": ([vp, vp, i], i),
        "pmhd_get_state": ([vp, vp, i], i),
        "pmhd_set_time": ([vp, d, ctypes.c_longlong], i),
        "pmhd_advance": ([vp, d, ctypes.c_longlong, P(Stats)], i),
        "pmhd_get_stats": ([vp, P(Stats)], i),
        "pmhd_diagnostics": ([vp, P(d)], i),
        "pmhd_write_dat": ([vp, ctypes.c_char_p, ctypes.c_char_p], i),
        "pmhd_dat_filename": ([vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t], i),
        "pmhd_strerror": ([i], ctypes.c_char_p),
        "pmhd_get_config": ([vp, P(Config)], i),
        "pmhd_problem_state": ([P(Config), i, P(d), i, vp], i),
        "pmhd_advance_noalloc": ([P(Config), vp, vp, d, ctypes.c_longlong, d, ctypes.c_longlong, vp, P(Stats)], i),
        "pmhd_ensemble_describe_default": ([i, ctypes.c_ulonglong, P(MemberDesc)], i),
        "pmhd_ensemble_create": ([P(Config), P(MemberDesc), i, P(vp)], i),
        "pmhd_ensemble_advance": ([vp, ctypes.c_longlong, P(Stats)], i),
        "pmhd_ensemble_member_stats": ([vp, i, P(Stats)], i),
        "pmhd_ensemble_get_state": ([vp, i, vp, i], i),
        "pmhd_ensemble_destroy": ([vp], i),
        "pmhd_conv3x3": ([i, vp, i, i, i, i, vp, P(ctypes.c_float), i, vp, vp, vp, vp], i),
        "pmhd_conv3x3_wgrad": ([vp, vp, i, i, i, i, i, P(ctypes.c_float), P(ctypes.c_float), vp], i),
        "pmhd_learned_loss_grad": ([vp, vp, i, i, i, ctypes.c_float, ctypes.c_float, vp, P(d), vp], i),
        "pmhd_learned_config_default": ([P(LearnedConfig)], i),
        "pmhd_learned_create": ([P(LearnedConfig), P(vp)], i),
        "pmhd_learned_destroy": ([vp], i),
        "pmhd_learned_generate": ([vp, i, P(d), i, d, i, P(i)], i),
        "pmhd_learned_generate_rollout": ([vp, i, P(d), i, d, i, P(i)], i),
        "pmhd_learned_generate_corrected": ([vp, i, P(d), i, d, i, P(i)], i),
        "pmhd_learned_num_pairs": ([vp], i),
        "pmhd_learned_train": ([vp, i, i, d, P(ctypes.c_float)], i),
        "pmhd_learned_run": ([vp, i, P(d), i, d, i, P(d), P(LearnedStats)], i),
        "pmhd_learned_fine_run": ([vp, i, P(d), i, d, i, P(d), P(LearnedStats)], i),
        "pmhd_learned_save": ([vp, ctypes.c_char_p], i),
        "pmhd_learned_load": ([vp, ctypes.c_char_p], i),
        "pmhd_euler2d_create": ([i, i, i, i, i, i, i, P(vp)], i),
        "pmhd_euler2d_advance": ([vp, d, ctypes.c_longlong, P(EulerStats)], i),
        "pmhd_euler2d_get_prim": ([vp, vp], i),
        "pmhd_euler2d_destroy": ([vp], i),
        "pmhd_euler1d_run": ([i, i, i, i, i, i, vp, P(EulerStats)], i),
        "pmhd_write_restart": ([vp, ctypes.c_char_p], i),
        "pmhd_read_restart": ([vp, ctypes.c_char_p], i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def strerror(status):
    return load().pmhd_strerror(status).decode()


def default_config():
    c = Config()
    load().pmhd_config_default(ctypes.byref(c))
    return c


def problem_state(problem, params=None, **cfg_kwargs):
    """Host-only initial state (ghosted AoS) of `problem` for the
    configuration Solver(**cfg_kwargs) would use; needs no GPU."""
    c = make_config(**cfg_kwargs)
    dt = np.float32 if c.precision == FP32 else np.float64
    U = np.empty((c.ny + 4, c.nx + 4, 9), dtype=dt)
    arr, n = None, 0
    if params is not None:
        n = len(params)
        arr = (ctypes.c_double * n)(*params)
    _check(load().pmhd_problem_state(ctypes.byref(c), problem, arr, n, U.ctypes.data), "pmhd_problem_state")
    return U


def make_config(nx=128, ny=128, precision="fp64", exact=False, order="muscl", solver="hlld", cfl=0.25,
                alpha=0.18, gamma=5.0 / 3.0, hlld_tol=1e-4, domain=(0.0, 1.0, 0.0, 1.0), bc=(0, 0, 0, 0),
                device=0, steps_per_graph=0, autotune=False):
    c = default_config()
    c.nx, c.ny = nx, ny
    c.x_min, c.x_max, c.y_min, c.y_max = domain
    c.gamma, c.hlld_tol, c.cfl, c.alpha = gamma, hlld_tol, cfl, alpha
    c.order = {"muscl": ORDER_MUSCL, "first": ORDER_FIRST, "hancock": ORDER_HANCOCK}[order]
    c.solver = SOLVER_HLLD if solver == "hlld" else SOLVER_HLL
    c.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    c.exact = int(bool(exact))
    for k in range(4):
        c.bc[k] = bc[k]
    c.device = device
    c.steps_per_graph = steps_per_graph
    c.autotune = int(bool(autotune))
    return c


def _check(status, where):
    if status != OK:
        raise PmhdError(status, where)


class Solver:
    """One grid on one GPU (a pmhd_solver handle)."""

    def __init__(self, nx=128, ny=128, precision="fp64", exact=False, order="muscl",
                 solver="hlld", cfl=0.25, alpha=0.18, gamma=5.0 / 3.0, hlld_tol=1e-4,
                 domain=(0.0, 1.0, 0.0, 1.0), bc=(0, 0, 0, 0), device=0, steps_per_graph=0, autotune=False):
        L = load()
        c = make_config(nx, ny, precision, exact, order, solver, cfl, alpha, gamma, hlld_tol, domain, bc,
                        device, steps_per_graph, autotune)
        self.cfg = c
        self.dtype = np.float32 if c.precision == FP32 else np.float64
        h = ctypes.c_void_p()
        _check(L.pmhd_create(ctypes.byref(c), ctypes.byref(h)), "pmhd_create")
        self._h = h

    # context manager / lifetime
    def close(self):
        if getattr(self, "_h", None):
            load().pmhd_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _shape(self, layout):
        c = self.cfg
        return (c.ny, c.nx, 9) if layout == LAYOUT_INTERIOR else (c.ny + 4, c.nx + 4, 9)

    def init_problem(self, problem, params=None):
        arr = None
        n = 0
        if params is not None:
            n = len(params)
            arr = (ctypes.c_double * n)(*params)
        _check(load().pmhd_init_problem(self._h, problem, arr, n), "pmhd_init_problem")

    def set_state(self, U, layout=LAYOUT_INTERIOR):
        U = np.ascontiguousarray(U, dtype=self.dtype)
        assert U.shape == self._shape(layout), (U.shape, self._shape(layout))
        _check(load().pmhd_set_state(self._h, U.ctypes.data, layout), "pmhd_set_state")

    def get_state(self, layout=LAYOUT_INTERIOR, out=None):
        if out is None:
            out = np.empty(self._shape(layout), dtype=self.dtype)
        assert out.shape == self._shape(layout) and out.dtype == self.dtype and out.flags["C_CONTIGUOUS"]
        _check(load().pmhd_get_state(self._h, out.ctypes.data, layout), "pmhd_get_state")
        return out

    def set_time(self, t, steps=0):
        _check(load().pmhd_set_time(self._h, t, steps), "pmhd_set_time")

    def advance(self, t_end=float("inf"), max_steps=-1, check=True):
        st = Stats()
        rc = load().pmhd_advance(self._h, t_end, max_steps, ctypes.byref(st))
        if check:
            _check(rc, "pmhd_advance")
        return st

    def stats(self):
        st = Stats()
        _check(load().pmhd_get_stats(self._h, ctypes.byref(st)), "pmhd_get_stats")
        return st

    def diagnostics(self):
        out = (ctypes.c_double * 3)()
        _check(load().pmhd_diagnostics(self._h, out), "pmhd_diagnostics")
        return tuple(out)

    def write_dat(self, path, title=None):
        _check(load().pmhd_write_dat(self._h, path.encode(), title.encode() if title else None),
               "pmhd_write_dat")

    def write_restart(self, path):
        _check(load().pmhd_write_restart(self._h, path.encode()), "pmhd_write_restart")

    def read_restart(self, path):
        _check(load().pmhd_read_restart(self._h, path.encode()), "pmhd_read_restart")

    def dat_filename(self, prob_base="orszag_tang"):
        buf = ctypes.create_string_buffer(512)
        _check(load().pmhd_dat_filename(self._h, prob_base.encode(), buf, 512), "pmhd_dat_filename")
        return buf.value.decode()


def describe_ensemble(n, seed=0):
    """The benchmark ensemble (pmhd_ensemble_describe_default): a ctypes
    array of n MemberDesc; needs no GPU."""
    arr = (MemberDesc * n)()
    _check(load().pmhd_ensemble_describe_default(n, seed, arr), "pmhd_ensemble_describe_default")
    return arr


def member(nx, ny, problem=PROBLEM_ORSZAG_TANG, params=(), t_end=0.5, gamma=5.0 / 3.0,
           domain=(0.0, 1.0, 0.0, 1.0), bc=(0, 0, 0, 0)):
    """One MemberDesc from keyword arguments."""
    m = MemberDesc()
    m.nx, m.ny = nx, ny
    m.x_min, m.x_max, m.y_min, m.y_max = domain
    m.gamma = gamma
    for k in range(4):
        m.bc[k] = bc[k]
    m.problem = problem
    m.nparams = len(params)
    for k, v in enumerate(params):
        m.params[k] = v
    m.t_end = t_end
    return m


class Ensemble:
    """Many independent grids advanced by the same launches (a pmhd_ensemble
    handle).  `members` is a sequence (or ctypes array) of MemberDesc; the
    keyword arguments give the common configuration as for Solver."""

    def __init__(self, members, precision="fp64", exact=False, order="muscl", solver="hlld", cfl=0.25,
                 alpha=0.18, hlld_tol=1e-4, device=0, steps_per_graph=0, autotune=False):
        L = load()
        n = len(members)
        arr = members if isinstance(members, ctypes.Array) else (MemberDesc * n)(*members)
        self.members = arr
        c = make_config(precision=precision, exact=exact, order=order, solver=solver, cfl=cfl, alpha=alpha,
                        hlld_tol=hlld_tol, device=device, steps_per_graph=steps_per_graph, autotune=autotune)
        self.cfg = c
        self.dtype = np.float32 if c.precision == FP32 else np.float64
        h = ctypes.c_void_p()
        _check(L.pmhd_ensemble_create(ctypes.byref(c), arr, n, ctypes.byref(h)), "pmhd_ensemble_create")
        self._h = h

    def __len__(self):
        return len(self.members)

    def close(self):
        if getattr(self, "_h", None):
            load().pmhd_ensemble_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def advance(self, max_steps=-1, check=True):
        st = Stats()
        rc = load().pmhd_ensemble_advance(self._h, max_steps, ctypes.byref(st))
        if check:
            _check(rc, "pmhd_ensemble_advance")
        return st

    def member_stats(self, k):
        st = Stats()
        _check(load().pmhd_ensemble_member_stats(self._h, k, ctypes.byref(st)), "pmhd_ensemble_member_stats")
        return st

    def get_state(self, k, layout=LAYOUT_INTERIOR):
        m = self.members[k]
        shape = (m.ny, m.nx, 9) if layout == LAYOUT_INTERIOR else (m.ny + 4, m.nx + 4, 9)
        out = np.empty(shape, dtype=self.dtype)
        _check(load().pmhd_ensemble_get_state(self._h, k, out.ctypes.data, layout), "pmhd_ensemble_get_state")
        return out


def _params_arg(params):
    if params is None or len(params) == 0:
        return None, 0
    return (ctypes.c_double * len(params))(*params), len(params)


class Learned:
    """Learned coarse-grid correction (a pmhd_learned handle): training pairs
    from the solver, device training, corrected and plain coarse runs, and
    the fine run they are measured against."""

    def __init__(self, **kw):
        L = load()
        c = LearnedConfig()
        _check(L.pmhd_learned_config_default(ctypes.byref(c)), "pmhd_learned_config_default")
        for k, val in kw.items():
            if k == "precision" and isinstance(val, str):
                val = PRECISIONS[val]
            if k == "domain":
                c.x_min, c.x_max, c.y_min, c.y_max = val
                continue
            setattr(c, k, val)
        self.cfg = c
        h = ctypes.c_void_p()
        _check(L.pmhd_learned_create(ctypes.byref(c), ctypes.byref(h)), "pmhd_learned_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            load().pmhd_learned_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_pairs(self):
        return load().pmhd_learned_num_pairs(self._h)

    def generate(self, problem=PROBLEM_ORSZAG_TANG, params=None, t_end=0.5, every=1, rollout=False,
                 corrected=False):
        """Training pairs; rollout=True takes them along the plain coarse
        trajectory (pmhd_learned_generate_rollout), corrected=True along the
        trajectory the current network corrects (pmhd_learned_generate_corrected)."""
        arr, n = _params_arg(params)
        added = ctypes.c_int()
        fn = ("pmhd_learned_generate_corrected" if corrected else
              "pmhd_learned_generate_rollout" if rollout else "pmhd_learned_generate")
        _check(getattr(load(), fn)(self._h, problem, arr, n, t_end, every, ctypes.byref(added)), fn)
        return added.value

    def train(self, iters=1000, batch=8, lr=2e-3):
        losses = (ctypes.c_float * iters)()
        _check(load().pmhd_learned_train(self._h, iters, batch, lr, losses), "pmhd_learned_train")
        return np.frombuffer(losses, dtype=np.float32).copy()

    def run(self, problem=PROBLEM_ORSZAG_TANG, params=None, t_end=0.5, use_net=True):
        arr, n = _params_arg(params)
        out = np.empty((self.cfg.ny, self.cfg.nx, 9), dtype=np.float64)
        st = LearnedStats()
        _check(load().pmhd_learned_run(self._h, problem, arr, n, t_end, int(bool(use_net)),
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(st)),
               "pmhd_learned_run")
        return out, st

    def fine_run(self, problem=PROBLEM_ORSZAG_TANG, params=None, t_end=0.5, refine=4):
        arr, n = _params_arg(params)
        out = np.empty((self.cfg.ny, self.cfg.nx, 9), dtype=np.float64)
        st = LearnedStats()
        _check(load().pmhd_learned_fine_run(self._h, problem, arr, n, t_end, refine,
                                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(st)),
               "pmhd_learned_fine_run")
        return out, st

    def save(self, path):
        _check(load().pmhd_learned_save(self._h, path.encode()), "pmhd_learned_save")

    def load_weights(self, path):
        _check(load().pmhd_learned_load(self._h, path.encode()), "pmhd_learned_load")


def _euler_solver(solver):
    return SOLVER_HLL if solver == "hll" else SOLVER_HLLC


EULER_SHOCK_BUBBLE = 100  # PMHD_EULER_SHOCK_BUBBLE


class Euler2D:
    """The Euler sibling's 2D problems (a pmhd_euler2d handle): Liska-Wendroff
    configuration 3, 6 or 12 on an nx x ny grid of [0,1]^2
    (src/euler/riemann2d_cpu.cpp), or config="shock_bubble" (EULER_SHOCK_BUBBLE):
    the Haas-Sturtevant shock-bubble program (src/euler/euler2d_cpu.cpp) on
    nx x ny cells of its 0.225 x 0.089 m domain (the reference's grid is
    500 x 197, the default here)."""

    def __init__(self, nx=None, ny=None, config=3, solver="hllc", precision="fp64", exact=False, device=0):
        if config == "shock_bubble":
            config = EULER_SHOCK_BUBBLE
        if config == EULER_SHOCK_BUBBLE:
            nx = 500 if nx is None else nx
            ny = 197 if ny is None else ny
        ny = nx if ny is None else ny
        self.nx, self.ny, self.config, self.precision = nx, ny, config, precision
        self.dtype = np.float32 if precision == "fp32" else np.float64
        self.steps, self.t = 0, 0.0
        h = ctypes.c_void_p()
        _check(load().pmhd_euler2d_create(nx, ny, config, _euler_solver(solver), PRECISIONS[precision],
                                          int(bool(exact)), device, ctypes.byref(h)), "pmhd_euler2d_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            load().pmhd_euler2d_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def advance(self, t_end=-1.0, max_steps=-1):
        st = EulerStats()
        _check(load().pmhd_euler2d_advance(self._h, t_end, max_steps, ctypes.byref(st)), "pmhd_euler2d_advance")
        self.steps, self.t = st.steps, st.t
        return st

    def prims(self):
        out = np.empty((self.ny, self.nx, 4), dtype=self.dtype)
        _check(load().pmhd_euler2d_get_prim(self._h, out.ctypes.data), "pmhd_euler2d_get_prim")
        return out

    def write_dat(self, path):
        """Writes the state as the shock-bubble program's .dat file
        (src/euler/euler2d_cpu.cpp:375-395): three '#' header lines (time,
        steps, end time), then x outermost, one 'x y rho u v p' line per cell in
        scientific notation with max_digits10 digits, a blank line after each
        column; cell centres are binary64 expressions stored in the
        precision's type, as there.  Returns path."""
        if self.config != EULER_SHOCK_BUBBLE:
            raise PmhdError(ERR_ARG, "write_dat (the .dat layout is the shock-bubble program's)")
        T = self.dtype
        f = "%.9e" if T == np.float32 else "%.17e"
        dx = float(T(T(0.225 - 0.0) / T(self.nx)))
        dy = float(T(T(0.089 - 0.0) / T(self.ny)))
        w = self.prims()
        ys = [f % float(T(0.0 + (j + 0.5) * dy)) for j in range(self.ny)]
        with open(path, "w") as out:
            out.write("# Time = %s\n# Steps = %d\n# T_END = %s\n" % (f % float(T(self.t)), self.steps, f % 0.0011741))
            for i in range(self.nx):
                x = f % float(T(0.0 + (i + 0.5) * dx))
                col = w[:, i, :]
                out.write("".join(x + " " + ys[j] + " " + " ".join(f % float(v) for v in col[j]) + "\n"
                                  for j in range(self.ny)))
                out.write("\n")
        return path


def euler1d(n, test, solver="hllc", precision="fp64", exact=False, device=0):
    """Toro test `test` on n cells: (EulerStats, [n][3] = rho, u, p)."""
    out = np.empty((n, 3), dtype=np.float32 if precision == "fp32" else np.float64)
    st = EulerStats()
    _check(load().pmhd_euler1d_run(n, test, _euler_solver(solver), PRECISIONS[precision], int(bool(exact)), device,
                                   out.ctypes.data, ctypes.byref(st)), "pmhd_euler1d_run")
    return st, out


def relative_l2(ref, other):
    """Per-variable relative L2 = RMS(ref - other) / RMS(ref), the metric of
    the reference's analysis/mhd/compare_precision.py:51-58, over the last
    axis of (..., nvar) arrays."""
    ref = np.asarray(ref, dtype=np.float64).reshape(-1, ref.shape[-1])
    other = np.asarray(other, dtype=np.float64).reshape(-1, ref.shape[-1])
    d = ref - other
    l2 = np.sqrt(np.mean(d * d, axis=0))
    rms = np.sqrt(np.mean(ref * ref, axis=0))
    return np.where(rms > 0, l2 / np.where(rms > 0, rms, 1.0), 0.0)


def conserved_to_dat_columns(U, gamma=5.0 / 3.0):
    """Primitive columns (rho vx vy vz p Bx By Bz E) of a (..., 9) conserved
    array, as the reference .dat file lists them."""
    U = np.asarray(U, dtype=np.float64)
    rho = np.maximum(U[..., 0], 1e-12)
    vx, vy, vz = U[..., 1] / rho, U[..., 2] / rho, U[..., 3] / rho
    bx, by, bz = U[..., 5], U[..., 6], U[..., 7]
    p = (gamma - 1.0) * (U[..., 4] - 0.5 * rho * (vx * vx + vy * vy + vz * vz) - 0.5 * (bx * bx + by * by + bz * bz))
    return np.stack([rho, vx, vy, vz, p, bx, by, bz, U[..., 4]], axis=-1)
