"""
ctypes binding of ``libcms_b200.so`` (C ABI in ``include/cms_b200.h``).

The library is built in-tree (``cms-cuda_b200/build.py``) and loaded from
this directory.  There is no CPU fallback: if the library or a GPU is
missing, calls fail loudly.
"""

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcms_b200.so")

CMS_HOST, CMS_DEVICE = 0, 1
OK, ERR_ARG, ERR_CUDA, ERR_STATE, ERR_COINCIDENT, ERR_EMPTY, ERR_CAPACITY = 0, -1, -2, -3, -4, -5, -6
ST_COINCIDENT, ST_EMPTY, ST_OVERFLOW, ST_NEAR_OVERFLOW = 1, 2, 4, 8
SC_FIELDS, SC_SIDE_FIELDS = 5, 7

# every symbol the header declares
EXPORTED = (
    "cms_ctx_create", "cms_ctx_destroy", "cms_set_settings", "cms_get_settings", "cms_load_batch",
    "cms_generate_surfaces", "cms_contact_ms", "cms_max_contact_ms", "cms_shape_complementarity",
    "cms_complex_info_get", "cms_export_atoms", "cms_export_neighbors", "cms_export_toroid",
    "cms_export_probes", "cms_export_dots", "cms_export_trimmed", "cms_run_graph", "cms_kernel_launches",
    "cms_last_error", "cms_version", "cms_device_count", "cms_profile_stages", "cms_stage_name",
    "cms_graph_launch", "cms_graph_check", "cms_nn_work", "cms_transfer_bytes", "cms_fp32_peak",
    "cms_nearest_dots", "cms_nearest_dots_noalloc", "cms_contact_ms_backward", "cms_set_backward",
    "cms_set_grad_total", "cms_grad_xyz", "cms_recompute_dots", "cms_export_dot_units",
    "cms_set_nn_variants", "cms_get_nn_variants", "cms_set_autotune", "cms_refine_begin",
    "cms_refine_set_params", "cms_refine_run", "cms_refine_pose", "cms_refine_end", "cms_residue_sums",
    "cms_nn_evaluated", "cms_set_surface_variants", "cms_get_surface_variants", "cms_set_concurrency",
)

NN_VARIANT_NAMES = ("q4 warp blocks", "q4 r512", "q2 warp blocks", "q2 r512")
SURFACE_STAGES = ("toroidal_count", "toroidal_emit", "concave_count", "concave_emit", "triples_count")
SURFACE_VARIANTS = 3
# cms_set_concurrency bits (CMS_CONC_* of the C header)
CONC_COUNT, CONC_EMIT, CONC_READOUT = 1, 2, 4
SURFACE_VARIANT_NAMES = {"toroidal": ("16 pairs x 4 warps", "32 pairs x 2 warps", "16 pairs x 4 warps, 6 CTAs/SM"),
                         "concave": ("4 CTAs/SM", "5 CTAs/SM", "6 CTAs/SM"),
                         "triples": ("rows <= 128 cached", "rows <= 64 cached, 10 CTAs/SM",
                                     "rows <= 64 cached, 12 CTAs/SM")}


class Settings(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("rp", "density", "band", "sep", "weight", "binwidth_dist", "binwidth_norm")]


class ComplexInfo(ctypes.Structure):
    _fields_ = [
        ("n_atoms", ctypes.c_int64), ("n_binder", ctypes.c_int64),
        ("nb_entries", ctypes.c_int64), ("bu_entries", ctypes.c_int64),
        ("max_nb", ctypes.c_int64), ("max_bu", ctypes.c_int64),
        ("n_toroid", ctypes.c_int64), ("n_probes", ctypes.c_int64),
        ("n_probes_plus", ctypes.c_int64 * 2), ("n_probes_minus", ctypes.c_int64 * 2),
        ("n_dots", ctypes.c_int64 * 2), ("n_trimmed", ctypes.c_int64 * 2),
        ("convex", ctypes.c_int64), ("toroidal", ctypes.c_int64), ("concave", ctypes.c_int64),
        ("n_blocked", ctypes.c_int64 * 2), ("n_attended", ctypes.c_int64 * 2),
        ("status", ctypes.c_int32), ("coincident_i", ctypes.c_int32), ("coincident_j", ctypes.c_int32),
        ("radmax", ctypes.c_double),
    ]


class CmsError(RuntimeError):
    """Error reported by the CUDA library."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


_lib = None
_lock = threading.Lock()

_VP = ctypes.c_void_p
_I32 = ctypes.c_int32
_PI64 = ctypes.POINTER(ctypes.c_int64)


def load():
    """Load the CUDA library once; raises OSError when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with `python cms-cuda_b200/build.py`")
        lib = ctypes.CDLL(LIB_PATH)
        sig = {
            "cms_ctx_create": [ctypes.POINTER(_VP), ctypes.c_int, _VP],
            "cms_ctx_destroy": [_VP],
            "cms_set_settings": [_VP, ctypes.POINTER(Settings)],
            "cms_get_settings": [_VP, ctypes.POINTER(Settings)],
            "cms_load_batch": [_VP, _I32, _PI64, _PI64, _VP, _VP, _VP, _I32],
            "cms_generate_surfaces": [_VP, _I32],
            "cms_contact_ms": [_VP, _VP, _VP, _I32],
            "cms_max_contact_ms": [_VP, _VP, _VP, _I32],
            "cms_shape_complementarity": [_VP, _VP, _VP, _I32],
            "cms_complex_info_get": [_VP, _I32, ctypes.POINTER(ComplexInfo)],
            "cms_export_atoms": [_VP, _I32, _VP, _VP, _VP, _VP],
            "cms_export_neighbors": [_VP, _I32, _VP, _VP, _VP, _VP],
            "cms_export_toroid": [_VP, _I32, _VP, _VP, _VP, _VP, _VP, _VP],
            "cms_export_probes": [_VP, _I32, _VP, _VP, _VP, _VP, _VP, _VP],
            "cms_export_dots": [_VP, _I32, _I32, _VP, _VP, _VP, _VP, _VP, _VP],
            "cms_export_trimmed": [_VP, _I32, _I32, _VP],
            "cms_run_graph": [_VP],
            "cms_graph_launch": [_VP],
            "cms_graph_check": [_VP],
            "cms_nn_work": [_VP, _PI64],
            "cms_transfer_bytes": [_VP, _PI64, _PI64],
            "cms_fp32_peak": [_VP, ctypes.POINTER(ctypes.c_double)],
            "cms_nearest_dots": [_VP, _VP, ctypes.c_int64, _VP, ctypes.c_int64, _VP, _VP, _I32],
            "cms_contact_ms_backward": [_VP, _I32, _VP, _VP, _I32],
            "cms_set_backward": [_VP, _I32, _I32],
            "cms_set_grad_total": [_VP, _VP, _I32],
            "cms_grad_xyz": [_VP, _VP, _I32],
            "cms_recompute_dots": [_VP, _I32, _I32, _VP, _VP],
            "cms_export_dot_units": [_VP, _I32, _I32, _VP, _VP],
            "cms_set_nn_variants": [_VP, _VP],
            "cms_get_nn_variants": [_VP, _VP, _VP],
            "cms_set_autotune": [_VP, _I32],
            "cms_refine_begin": [_VP, _VP, _I32, _I32],
            "cms_refine_set_params": [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double],
            "cms_refine_run": [_VP, _I32, _VP, _I32],
            "cms_refine_pose": [_VP, _VP, _VP, _VP, _I32],
            "cms_refine_end": [_VP],
            "cms_residue_sums": [_VP, _I32, ctypes.c_int64, _PI64, ctypes.c_int64, _VP, _VP, _I32],
            "cms_nn_evaluated": [_VP, _PI64],
            "cms_set_surface_variants": [_VP, _VP],
            "cms_get_surface_variants": [_VP, _VP, _VP],
            "cms_set_concurrency": [_VP, _I32],
        }
        for name, args in sig.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = ctypes.c_int32
        lib.cms_kernel_launches.argtypes = [_VP]
        lib.cms_kernel_launches.restype = ctypes.c_int64
        lib.cms_last_error.argtypes = [_VP]
        lib.cms_last_error.restype = ctypes.c_char_p
        lib.cms_version.argtypes = []
        lib.cms_version.restype = ctypes.c_char_p
        lib.cms_device_count.argtypes = []
        lib.cms_device_count.restype = ctypes.c_int32
        lib.cms_profile_stages.argtypes = [_VP, _VP, _I32, ctypes.POINTER(_I32)]
        lib.cms_profile_stages.restype = ctypes.c_int32
        lib.cms_stage_name.argtypes = [_I32]
        lib.cms_stage_name.restype = ctypes.c_char_p
        _lib = lib
        return lib


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class Context:
    """One device context (one CUDA stream) of the library; not thread-safe."""

    def __init__(self, device=0, stream=None):
        self.lib = load()
        h = ctypes.c_void_p()
        st = self.lib.cms_ctx_create(ctypes.byref(h), int(device), ctypes.c_void_p(stream) if stream else None)
        self.h = h
        self._check(st)
        self.device = int(device)
        self.B = 0
        self.N = 0

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.h.value:
                self.lib.cms_ctx_destroy(self.h)
                self.h = ctypes.c_void_p()
        except Exception:
            pass

    def close(self):
        self.__del__()

    def _check(self, status):
        if status != OK:
            msg = self.lib.cms_last_error(self.h).decode() if self.h.value else "context creation failed"
            raise CmsError(status, msg)

    # -- settings / inputs ----------------------------------------------------
    def set_settings(self, s):
        v = Settings(float(s.rp), float(s.density), float(s.band), float(s.sep), float(s.weight),
                     float(s.binwidth_dist), float(s.binwidth_norm))
        self._check(self.lib.cms_set_settings(self.h, ctypes.byref(v)))

    def load_batch(self, atom_off, n_binder, xyz, radius, density=None):
        atom_off = np.ascontiguousarray(atom_off, dtype=np.int64)
        n_binder = np.ascontiguousarray(n_binder, dtype=np.int64)
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        radius = np.ascontiguousarray(radius, dtype=np.float64)
        if density is not None:
            density = np.ascontiguousarray(density, dtype=np.float64)
        B = len(n_binder)
        if len(atom_off) != B + 1 or atom_off[-1] != len(radius) or len(xyz) != len(radius):
            raise ValueError("inconsistent batch arrays")
        self._check(self.lib.cms_load_batch(self.h, B, atom_off.ctypes.data_as(_PI64),
                                            n_binder.ctypes.data_as(_PI64), _ptr(xyz), _ptr(radius),
                                            _ptr(density), CMS_HOST))
        self.B, self.N = B, int(atom_off[-1])

    def load_batch_device(self, atom_off, n_binder, xyz_ptr, radius_ptr, density_ptr=None):
        """Device-pointer variant (e.g. torch tensors' data_ptr())."""
        atom_off = np.ascontiguousarray(atom_off, dtype=np.int64)
        n_binder = np.ascontiguousarray(n_binder, dtype=np.int64)
        self._check(self.lib.cms_load_batch(self.h, len(n_binder), atom_off.ctypes.data_as(_PI64),
                                            n_binder.ctypes.data_as(_PI64), ctypes.c_void_p(xyz_ptr),
                                            ctypes.c_void_p(radius_ptr),
                                            ctypes.c_void_p(density_ptr) if density_ptr else None, CMS_DEVICE))
        self.B, self.N = len(n_binder), int(atom_off[-1])

    # -- pipeline -------------------------------------------------------------
    def generate(self, all_atoms=False):
        self._check(self.lib.cms_generate_surfaces(self.h, 1 if all_atoms else 0))

    def run_graph(self):
        self._check(self.lib.cms_run_graph(self.h))

    def graph_launch(self):
        """Replay the captured pipeline asynchronously on the context's stream."""
        self._check(self.lib.cms_graph_launch(self.h))

    def graph_check(self):
        self._check(self.lib.cms_graph_check(self.h))

    def set_nn_variants(self, variants):
        """Force the three search shapes (CMS, SC band, SC argmin); turns the autotuner off."""
        v = np.ascontiguousarray(variants, dtype=np.int32)
        self._check(self.lib.cms_set_nn_variants(self.h, _ptr(v)))

    def set_surface_variants(self, variants):
        """Force the surface kernels' shapes (toroidal count / emit, concave count / emit, triple count); turns
        the tuner off."""
        v = np.ascontiguousarray(variants, dtype=np.int32)
        self._check(self.lib.cms_set_surface_variants(self.h, _ptr(v)))

    def surface_variants(self):
        """(shape per tuned surface stage, measured ms per stage and shape) of the autotuner."""
        v = np.zeros(len(SURFACE_STAGES), np.int32)
        ms = np.zeros(len(SURFACE_STAGES) * SURFACE_VARIANTS)
        self._check(self.lib.cms_get_surface_variants(self.h, _ptr(v), _ptr(ms)))
        return v.tolist(), ms.reshape(len(SURFACE_STAGES), SURFACE_VARIANTS)

    def set_concurrency(self, mode=True):
        """Stages run as parallel graph branches: an OR of CONC_COUNT, CONC_EMIT and CONC_READOUT
        (True: all three, False: every stage in order)."""
        if isinstance(mode, bool):
            mode = CONC_COUNT | CONC_EMIT | CONC_READOUT if mode else 0
        self._check(self.lib.cms_set_concurrency(self.h, int(mode)))

    def set_autotune(self, enable=True):
        self._check(self.lib.cms_set_autotune(self.h, 1 if enable else 0))

    def nn_variants(self):
        """(chosen shape per search, measured ms per search and shape) of the autotuner."""
        v = np.zeros(3, np.int32)
        ms = np.zeros(12)
        self._check(self.lib.cms_get_nn_variants(self.h, _ptr(v), _ptr(ms)))
        return v.tolist(), ms.reshape(3, 4)

    # -- pose refinement ------------------------------------------------------
    def refine_begin(self, ref_xyz, max_steps):
        x = np.ascontiguousarray(ref_xyz, dtype=np.float64).reshape(-1, 3)
        self._check(self.lib.cms_refine_begin(self.h, _ptr(x), int(max_steps), CMS_HOST))

    def refine_set_params(self, eta_t, eta_w, max_t, max_w):
        self._check(self.lib.cms_refine_set_params(self.h, float(eta_t), float(eta_w), float(max_t), float(max_w)))

    def refine_run(self, steps):
        """CMS (steps x B) of every evaluated pose."""
        h = np.empty((int(steps), self.B), dtype=np.float64)
        self._check(self.lib.cms_refine_run(self.h, int(steps), _ptr(h), CMS_HOST))
        return h

    def refine_pose(self, xyz=True):
        rot = np.empty((self.B, 3, 3)); tr = np.empty((self.B, 3))
        x = np.empty((self.N, 3)) if xyz else None
        self._check(self.lib.cms_refine_pose(self.h, _ptr(rot), _ptr(tr), _ptr(x), CMS_HOST))
        return rot, tr, x

    def refine_end(self):
        self._check(self.lib.cms_refine_end(self.h))

    def nn_work(self):
        w = np.zeros(6, dtype=np.int64)
        self._check(self.lib.cms_nn_work(self.h, w.ctypes.data_as(_PI64)))
        return dict(cms_pairs=int(w[0]), cms_queries=int(w[1]), band_pairs=int(w[2]), band_queries=int(w[3]),
                    sc_pairs=int(w[4]), sc_queries=int(w[5]))

    def nn_evaluated(self):
        """Pairs the FP32 filter evaluated after culling and FP64 rechecks, per search (one counted run)."""
        w = np.zeros(6, dtype=np.int64)
        self._check(self.lib.cms_nn_evaluated(self.h, w.ctypes.data_as(_PI64)))
        names = ("cms", "band", "sc")
        return {**{f"{n}_evaluated": int(w[k]) for k, n in enumerate(names)},
                **{f"{n}_rechecks": int(w[3 + k]) for k, n in enumerate(names)}}

    def kernel_launches(self):
        return int(self.lib.cms_kernel_launches(self.h))

    def profile_stages(self):
        """{stage name: milliseconds} of one pipeline run with an event after every stage."""
        ms = np.zeros(64)
        n = ctypes.c_int32(0)
        self._check(self.lib.cms_profile_stages(self.h, _ptr(ms), 64, ctypes.byref(n)))
        return {self.lib.cms_stage_name(i).decode(): float(ms[i]) for i in range(n.value)}

    def nearest_dots(self, query, ref):
        """(min squared distance, first index) of each query point over the reference points."""
        q = np.ascontiguousarray(query, dtype=np.float64).reshape(-1, 3)
        r = np.ascontiguousarray(ref, dtype=np.float64).reshape(-1, 3)
        d2 = np.empty(len(q)); idx = np.empty(len(q), np.int32)
        self._check(self.lib.cms_nearest_dots(self.h, _ptr(q), len(q), _ptr(r), len(r), _ptr(d2), _ptr(idx),
                                              CMS_HOST))
        return d2, idx

    def fp32_peak(self):
        v = ctypes.c_double(0)
        self._check(self.lib.cms_fp32_peak(self.h, ctypes.byref(v)))
        return v.value

    def transfer_bytes(self):
        a, b = ctypes.c_int64(0), ctypes.c_int64(0)
        self._check(self.lib.cms_transfer_bytes(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def contact_ms(self, per_atom=True):
        per_atom = np.empty(self.N, dtype=np.float64) if per_atom else None
        totals = np.empty(2 * self.B, dtype=np.float64)
        self._check(self.lib.cms_contact_ms(self.h, _ptr(per_atom), _ptr(totals), CMS_HOST))
        return per_atom, totals.reshape(self.B, 2)

    def contact_ms_backward(self, target_side=True, grad_total=None):
        """d(sum_c grad_total[c] * CMS_c)/d(xyz) (N x 3) for one side, dot topology held fixed."""
        g = None if grad_total is None else np.ascontiguousarray(grad_total, dtype=np.float64)
        if g is not None and g.shape != (self.B,):
            raise ValueError(f"grad_total must have shape ({self.B},)")
        out = np.empty((self.N, 3), dtype=np.float64)
        self._check(self.lib.cms_contact_ms_backward(self.h, 1 if target_side else 0, _ptr(g), _ptr(out), CMS_HOST))
        return out

    def contact_ms_backward_device(self, target_side, grad_total_ptr, grad_xyz_ptr):
        """Device-pointer variant: grad_total (B) and grad_xyz (N x 3) are device buffers."""
        self._check(self.lib.cms_contact_ms_backward(self.h, 1 if target_side else 0, ctypes.c_void_p(grad_total_ptr),
                                                     ctypes.c_void_p(grad_xyz_ptr), CMS_DEVICE))

    def set_backward(self, enable=True, target_side=True):
        """Include the gradient of one side's CMS in the captured pipeline (upstream ones)."""
        self._check(self.lib.cms_set_backward(self.h, 1 if enable else 0, 1 if target_side else 0))

    def set_grad_total(self, grad_total):
        g = np.ascontiguousarray(grad_total, dtype=np.float64)
        self._check(self.lib.cms_set_grad_total(self.h, _ptr(g), CMS_HOST))

    def grad_xyz(self, out=None):
        """The last run's gradient (N x 3); `out` (float64, C-contiguous, N x 3), e.g. a pinned
        buffer reused across steps, receives it instead of a new array."""
        if out is None:
            out = np.empty((self.N, 3), dtype=np.float64)
        elif out.dtype != np.float64 or out.shape != (self.N, 3) or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float64 array of shape ({self.N}, 3)")
        self._check(self.lib.cms_grad_xyz(self.h, _ptr(out), CMS_HOST))
        return out

    def grad_xyz_device(self, ptr):
        """The last run's gradient copied to device memory at `ptr` (N x 3 float64)."""
        self._check(self.lib.cms_grad_xyz(self.h, ctypes.c_void_p(ptr), CMS_DEVICE))

    def recompute_dots(self, c, m, info):
        """Dots of complex c, molecule m recomputed by the adjoint's geometry (self-check)."""
        n = max(info.n_dots[m], 1)
        coor = np.empty((n, 3)); area = np.empty(n)
        self._check(self.lib.cms_recompute_dots(self.h, int(c), int(m), _ptr(coor), _ptr(area)))
        k = info.n_dots[m]
        return coor[:k], area[:k]

    def max_contact_ms(self):
        per_atom = np.empty(self.N, dtype=np.float64)
        totals = np.empty(self.B, dtype=np.float64)
        self._check(self.lib.cms_max_contact_ms(self.h, _ptr(per_atom), _ptr(totals), CMS_HOST))
        return per_atom, totals

    def residue_sums(self, res_off, res_atoms, values="cms"):
        """
        Per-residue sums of the per-atom CMS ("cms") or maximum CMS ("max") on
        the device: residue r adds atoms res_atoms[res_off[r]:res_off[r+1]]
        (batch atom indices) in that order.
        """
        off = np.ascontiguousarray(res_off, dtype=np.int64)
        atoms = np.ascontiguousarray(res_atoms, dtype=np.int32)
        n = len(off) - 1
        out = np.empty(max(n, 0), dtype=np.float64)
        self._check(self.lib.cms_residue_sums(self.h, {"cms": 0, "max": 1}[values], n, off.ctypes.data_as(_PI64),
                                              len(atoms), _ptr(atoms), _ptr(out), CMS_HOST))
        return out

    def shape_complementarity(self):
        sc = np.empty(self.B * SC_FIELDS, dtype=np.float64)
        sides = np.empty(self.B * 2 * SC_SIDE_FIELDS, dtype=np.float64)
        self._check(self.lib.cms_shape_complementarity(self.h, _ptr(sc), _ptr(sides), CMS_HOST))
        return sc.reshape(self.B, SC_FIELDS), sides.reshape(self.B, 2, SC_SIDE_FIELDS)

    # -- exports --------------------------------------------------------------
    def info(self, c):
        i = ComplexInfo()
        self._check(self.lib.cms_complex_info_get(self.h, int(c), ctypes.byref(i)))
        return i

    def export_atoms(self, c, n):
        atten = np.empty(n, np.int8); access = np.empty(n, np.int8)
        nn = np.empty(n, np.int32); nb = np.empty(n, np.int32)
        self._check(self.lib.cms_export_atoms(self.h, int(c), _ptr(atten), _ptr(access), _ptr(nn), _ptr(nb)))
        return atten, access, nn, nb

    def export_neighbors(self, c, n, info):
        nb_off = np.empty(n + 1, np.int64); nb_id = np.empty(max(info.nb_entries, 1), np.int32)
        bu_off = np.empty(n + 1, np.int64); bu_id = np.empty(max(info.bu_entries, 1), np.int32)
        self._check(self.lib.cms_export_neighbors(self.h, int(c), _ptr(nb_off), _ptr(nb_id), _ptr(bu_off),
                                                  _ptr(bu_id)))
        return nb_off, nb_id[:info.nb_entries], bu_off, bu_id[:info.bu_entries]

    def export_toroid(self, c, info):
        n = info.n_toroid
        a1 = np.empty(max(n, 1), np.int32); a2 = np.empty(max(n, 1), np.int32)
        uij = np.empty((max(n, 1), 3)); tij = np.empty((max(n, 1), 3)); rij = np.empty(max(n, 1))
        bet = np.empty(max(n, 1), np.int8)
        self._check(self.lib.cms_export_toroid(self.h, int(c), _ptr(a1), _ptr(a2), _ptr(uij), _ptr(tij), _ptr(rij),
                                               _ptr(bet)))
        return a1[:n], a2[:n], uij[:n], tij[:n], rij[:n], bet[:n].astype(bool)

    def export_probes(self, c, info):
        n = max(info.n_probes, 1)
        a0 = np.empty(n, np.int32); a1 = np.empty(n, np.int32); a2 = np.empty(n, np.int32)
        h = np.empty(n); pt = np.empty((n, 3)); alt = np.empty((n, 3))
        self._check(self.lib.cms_export_probes(self.h, int(c), _ptr(a0), _ptr(a1), _ptr(a2), _ptr(h), _ptr(pt),
                                               _ptr(alt)))
        k = info.n_probes
        return a0[:k], a1[:k], a2[:k], h[:k], pt[:k], alt[:k]

    def export_dots(self, c, m, info):
        n = max(info.n_dots[m], 1)
        coor = np.empty((n, 3)); nml = np.empty((n, 3)); area = np.empty(n)
        bur = np.empty(n, np.int8); typ = np.empty(n, np.int8); atom = np.empty(n, np.int32)
        self._check(self.lib.cms_export_dots(self.h, int(c), int(m), _ptr(coor), _ptr(nml), _ptr(area), _ptr(bur),
                                             _ptr(typ), _ptr(atom)))
        k = info.n_dots[m]
        return coor[:k], nml[:k], area[:k], bur[:k], typ[:k], atom[:k]

    def export_dot_units(self, c, m, info):
        """(unit, sub) construction indices of complex c's dots of molecule m."""
        n = max(info.n_dots[m], 1)
        unit = np.empty(n, np.int32); sub = np.empty(n, np.int32)
        self._check(self.lib.cms_export_dot_units(self.h, int(c), int(m), _ptr(unit), _ptr(sub)))
        k = info.n_dots[m]
        return unit[:k], sub[:k]

    def export_trimmed(self, c, m, info):
        n = max(info.n_trimmed[m], 1)
        idx = np.empty(n, np.int32)
        self._check(self.lib.cms_export_trimmed(self.h, int(c), int(m), _ptr(idx)))
        return idx[:info.n_trimmed[m]]


# Contexts are expensive to create (stream, pinned staging, tens of device
# buffers) and keep their workspace between runs, so calculators borrow them
# from a per-thread, per-device pool and hand them back when released -- the
# role CuPy's per-stream memory pool plays for the reference's GPU calculator.
_pool = threading.local()


def acquire_context(device=0):
    free = getattr(_pool, "free", None)
    if free is None:
        free = _pool.free = {}
    lst = free.setdefault(int(device), [])
    return lst.pop() if lst else Context(device)


def release_context(ctx, device=0):
    free = getattr(_pool, "free", None)
    if free is None:
        free = _pool.free = {}
    lst = free.setdefault(int(device), [])
    if len(lst) < 4:
        lst.append(ctx)


def device_count():
    try:
        return int(load().cms_device_count())
    except OSError:
        return 0


def version():
    return load().cms_version().decode()
