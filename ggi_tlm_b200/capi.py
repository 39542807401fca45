"""ctypes binding of the C-ABI in include/tlm_gpu.h.

This is the host-side mirror of the reference's time-loop call
(``CALL run_TLM()``, SRC/GGI_TLM.F90:157): a caller hands over the arrays
its setup stage produced (see ``ggi_tlm_b200.problem.build_tables``), then
advances the mesh and reads back probe samples and DFT accumulators.

The CUDA library is required.  There is no CPU fallback: if
``_lib/libtlm_gpu.so`` is missing or no CUDA device is present, every entry
point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libtlm_gpu.so")

TLM_PRECISION_FP32 = 32
TLM_PRECISION_FP64 = 64
MAX_ORDER = 8

TLM_OK, TLM_E_BADARG, TLM_E_UNSUPPORTED, TLM_E_OOM, TLM_E_CUDA, TLM_E_STATE, TLM_E_TIMEOUT = 0, -1, -2, -3, -4, -5, -6
ERRORS = {-1: "TLM_E_BADARG", -2: "TLM_E_UNSUPPORTED", -3: "TLM_E_OOM", -4: "TLM_E_CUDA", -5: "TLM_E_STATE",
          -6: "TLM_E_TIMEOUT"}

# every symbol include/tlm_gpu.h declares (checked by the CPU test suite)
EXPORTS = [
    "tlm_gpu_create", "tlm_gpu_set_cells", "tlm_gpu_set_materials", "tlm_gpu_set_pml", "tlm_gpu_set_excitation",
    "tlm_gpu_set_faces", "tlm_gpu_set_huygens", "tlm_gpu_set_outputs", "tlm_gpu_set_dft", "tlm_gpu_run",
    "tlm_gpu_synchronize", "tlm_gpu_fetch_cell_output", "tlm_gpu_fetch_dft", "tlm_gpu_fetch_links",
    "tlm_gpu_set_stream", "tlm_gpu_set_timing", "tlm_gpu_last_run_time", "tlm_gpu_memory_bytes",
    "tlm_gpu_last_run_launches", "tlm_gpu_destroy", "tlm_gpu_last_error", "tlm_gpu_set_variant",
    "tlm_gpu_num_variants", "tlm_gpu_fetch_links_noalloc", "tlm_gpu_batch_create", "tlm_gpu_batch_set_variant",
    "tlm_gpu_batch_run", "tlm_gpu_batch_synchronize", "tlm_gpu_batch_last_run", "tlm_gpu_batch_destroy",
    "tlm_gpu_set_small_to_zero", "tlm_gpu_set_pml_sigma", "tlm_gpu_set_face_excitation",
    "tlm_gpu_set_face_excitation_side", "tlm_gpu_set_face_excitation_scale",
    "tlm_gpu_set_face_outputs", "tlm_gpu_fetch_face_output", "tlm_gpu_set_outer_huygens",
    "tlm_gpu_set_far_field", "tlm_gpu_fetch_far_field", "tlm_gpu_pool_release", "tlm_gpu_pool_cached_bytes",
    "tlm_gpu_prepare", "tlm_gpu_set_output_series", "tlm_gpu_set_volume_dft", "tlm_gpu_fetch_volume_dft",
    "tlm_gpu_set_output_surfaces", "tlm_gpu_fetch_output_surfaces", "tlm_gpu_set_rcs", "tlm_gpu_fetch_rcs",
    "tlm_gpu_set_output_volumes", "tlm_gpu_fetch_output_volumes", "tlm_gpu_set_sar_volumes",
    "tlm_gpu_fetch_sar_volumes", "tlm_gpu_set_power_surfaces", "tlm_gpu_fetch_power_surfaces",
    "tlm_gpu_set_mode_outputs", "tlm_gpu_fetch_mode_outputs", "tlm_gpu_set_face_materials",
    "tlm_gpu_set_thin_layers", "tlm_gpu_set_face_thin_layers", "tlm_gpu_set_wrap",
    "tlm_gpu_halo_bytes", "tlm_gpu_halo_get", "tlm_gpu_halo_put", "tlm_gpu_set_test_wait_pad",
    "tlm_gpu_set_dft_gate", "tlm_gpu_batch_set_members",
]


def output_surface_shapes(t: dict) -> list:
    """(n_output_steps, n_faces) of each time-domain output surface: the
    steps first..min(last, n_timesteps) every interval."""
    res = []
    ptr = t.get("osurf_face_ptr", [0])
    for k in range(int(t.get("n_osurf", 0))):
        first, last, every = int(t["osurf_first"][k]), int(t["osurf_last"][k]), int(t["osurf_interval"][k])
        hi = min(last, int(t["n_timesteps"]))
        res.append(((hi - first) // every + 1 if hi >= first else 0, int(ptr[k + 1] - ptr[k])))
    return res


class TLMError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class MeshDesc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("n_timesteps", C.c_int32),
                ("dl", C.c_double), ("dt", C.c_double), ("R", C.c_double * 6), ("precision", C.c_int32),
                ("device", C.c_int32)]


_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)
_lib = None


def load_library(path: Optional[str] = None):
    """Load libtlm_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library not built: {path} (run python -m ggi_tlm_b200.build)")
    lib = C.CDLL(path)
    i64, i32 = C.c_int64, C.c_int32
    sig = {
        "tlm_gpu_create": [C.POINTER(MeshDesc), C.POINTER(i64)],
        "tlm_gpu_set_cells": [i64, _i32p, i32, _i32p, _i32p, _i32p, _i32p],
        "tlm_gpu_set_materials": [i64, i32, _i32p, _i32p, _i32p, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p,
                                  _f64p, _f64p, _f64p, i32],
        "tlm_gpu_set_pml": [i64, i32, _f64p, i32, _i32p],
        "tlm_gpu_set_pml_sigma": [i64, i32, _f64p],
        "tlm_gpu_set_face_excitation": [i64, i32, _i32p, _i32p, _i32p, _i32p],
        "tlm_gpu_set_face_excitation_side": [i64, i32, _i32p],
        "tlm_gpu_set_face_excitation_scale": [i64, i32, _f64p],
        "tlm_gpu_set_face_outputs": [i64, i32, _i32p, _i32p, _i32p],
        "tlm_gpu_set_outer_huygens": [i64, i32, _i32p, _f64p, _f64p, _f64p, C.c_double, C.c_double, i32],
        "tlm_gpu_set_far_field": [i64, i32, _f64p, _i32p, _i32p, _i32p],
        "tlm_gpu_fetch_far_field": [i64, _f64p],
        "tlm_gpu_pool_release": [],
        "tlm_gpu_prepare": [i64],
        "tlm_gpu_pool_cached_bytes": [C.POINTER(i64)],
        "tlm_gpu_fetch_face_output": [i64, i32, i32, _f64p],
        "tlm_gpu_set_excitation": [i64, i32, i32, _f64p, _f64p, i32, _i32p, _i32p, _i32p, _i32p, i32],
        "tlm_gpu_set_faces": [i64, i32, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, i32, i32],
        "tlm_gpu_set_huygens": [i64, i32, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_double, C.c_double, i32],
        "tlm_gpu_set_outputs": [i64, i32],
        "tlm_gpu_set_output_series": [i64, i32, _i32p],
        "tlm_gpu_set_volume_dft": [i64, i32, _f64p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p],
        "tlm_gpu_fetch_volume_dft": [i64, _f64p],
        "tlm_gpu_set_output_surfaces": [i64, i32, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p],
        "tlm_gpu_fetch_output_surfaces": [i64, _f64p],
        "tlm_gpu_set_rcs": [i64, C.c_double, C.c_double, i32, i32, i32, i32, _i32p, _i32p, _f64p],
        "tlm_gpu_fetch_rcs": [i64, _f64p],
        "tlm_gpu_set_output_volumes": [i64, i32, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p],
        "tlm_gpu_fetch_output_volumes": [i64, _f64p],
        "tlm_gpu_set_sar_volumes": [i64, i32, _f64p, _i32p, _i32p],
        "tlm_gpu_fetch_sar_volumes": [i64, _f64p],
        "tlm_gpu_set_power_surfaces": [i64, i32, _f64p, _i32p, _i32p, _i32p],
        "tlm_gpu_fetch_power_surfaces": [i64, _f64p],
        "tlm_gpu_set_mode_outputs": [i64, i32, _i32p, _i32p, _i32p, _i32p, _f64p],
        "tlm_gpu_set_face_materials": [i64, i32, _i32p],
        "tlm_gpu_set_thin_layers": [i64, i32, _f64p, _f64p, _f64p, _i32p, i32],
        "tlm_gpu_set_face_thin_layers": [i64, i32, _i32p],
        "tlm_gpu_set_wrap": [i64, i32, i32, i32],
        "tlm_gpu_halo_bytes": [i64, C.POINTER(i64)],
        "tlm_gpu_set_test_wait_pad": [i64, i32],
        "tlm_gpu_set_dft_gate": [i64, i32, _i32p, _i32p, _i32p],
        "tlm_gpu_halo_get": [i64, i32, C.c_void_p],
        "tlm_gpu_halo_put": [i64, i32, C.c_void_p],
        "tlm_gpu_fetch_mode_outputs": [i64, i32, i32, _f64p],
        "tlm_gpu_set_small_to_zero": [i64, i32, C.c_double],
        "tlm_gpu_set_dft": [i64, i32, _f64p, _i32p, _i32p, _i32p, _i32p],
        "tlm_gpu_run": [i64, i32, i32],
        "tlm_gpu_synchronize": [i64],
        "tlm_gpu_fetch_cell_output": [i64, i32, i32, _f64p],
        "tlm_gpu_fetch_dft": [i64, _f64p],
        "tlm_gpu_fetch_links": [i64, _f64p],
        "tlm_gpu_fetch_links_noalloc": [i64, _f64p],
        "tlm_gpu_set_stream": [i64, C.c_void_p],
        "tlm_gpu_set_timing": [i64, i32],
        "tlm_gpu_last_run_time": [i64, C.POINTER(C.c_float), C.POINTER(C.c_float)],
        "tlm_gpu_memory_bytes": [i64, C.POINTER(i64)],
        "tlm_gpu_last_run_launches": [i64, C.POINTER(i64)],
        "tlm_gpu_destroy": [i64],
        "tlm_gpu_set_variant": [i64, i32],
        "tlm_gpu_num_variants": [C.POINTER(i32)],
        "tlm_gpu_last_error": [C.c_char_p, i32],
        "tlm_gpu_batch_create": [C.POINTER(i64), i32, C.POINTER(i64)],
        "tlm_gpu_batch_set_variant": [i64, i32],
        "tlm_gpu_batch_set_members": [i64, C.POINTER(i64), i32],
        "tlm_gpu_batch_run": [i64, i32],
        "tlm_gpu_batch_synchronize": [i64],
        "tlm_gpu_batch_last_run": [i64, C.POINTER(C.c_float), C.POINTER(i64), C.POINTER(i64)],
        "tlm_gpu_batch_destroy": [i64],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    _lib = lib
    return lib


def pool_cached_bytes() -> int:
    """Bytes the library's device-memory cache holds for reuse."""
    v = C.c_int64(0)
    _check(load_library().tlm_gpu_pool_cached_bytes(C.byref(v)))
    return int(v.value)


def pool_release():
    """Return every cached device block to the driver."""
    _check(load_library().tlm_gpu_pool_release())


def num_variants() -> int:
    n = C.c_int32(0)
    _check(load_library().tlm_gpu_num_variants(C.byref(n)))
    return n.value


def _check(rc: int):
    if rc != 0:
        buf = C.create_string_buffer(512)
        _lib.tlm_gpu_last_error(buf, 512)
        raise TLMError(rc, buf.value.decode(errors="replace"))


def _i32(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.int32).reshape(-1)
    return a if a.size else np.zeros(1, np.int32)


def _f64(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    return a if a.size else np.zeros(1, np.float64)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_i32p if a.dtype == np.int32 else _f64p)


class GpuMesh:
    """One mesh on the GPU, driven through the C-ABI exactly as the Fortran
    shim would drive it (create -> set_* -> run -> fetch -> destroy)."""

    def __init__(self, tables: dict, precision: int = TLM_PRECISION_FP64, device: int = 0):
        lib = load_library()
        t = tables
        self.t = t
        d = MeshDesc()
        d.nx, d.ny, d.nz, d.n_timesteps = t["nx"], t["ny"], t["nz"], t["n_timesteps"]
        d.dl, d.dt = t["dl"], t["dt"]
        d.R[:] = [float(v) for v in t["R"]]
        d.precision = precision
        d.device = device
        h = C.c_int64(0)
        _check(lib.tlm_gpu_create(C.byref(d), C.byref(h)))
        self.h = h.value
        self.precision = precision
        self.step = 0
        try:
            self._upload(t)
        except Exception:
            self.close()
            raise

    def _upload(self, t: dict):
        lib = _lib
        a = [_i32(t["cell_code"]), _i32(t["sp_material"]), _i32(t["sp_pml"]), _i32(t["sp_excitation"]),
             _i32(t["sp_output"])]
        _check(lib.tlm_gpu_set_cells(self.h, _p(a[0]), int(t["n_special"]), _p(a[1]), _p(a[2]), _p(a[3]), _p(a[4])))
        nm = int(t["n_materials"])
        if nm:
            m = [_i32(t[k]) for k in ("mat_type", "mat_eps_exists", "mat_mu_exists", "mat_eps_order", "mat_mu_order")]
            f = [_f64(t[k]) for k in ("mat_Ys_eps_f", "mat_Zs_mu_f", "mat_Ge", "mat_Rm", "mat_eps_a", "mat_eps_b",
                                      "mat_mu_a", "mat_mu_b")]
            stride = np.asarray(t["mat_eps_a"]).reshape(nm, -1).shape[1]
            _check(lib.tlm_gpu_set_materials(self.h, nm, *[_p(x) for x in m], *[_p(x) for x in f], stride))
        pp, pc = _f64(t["pml_params"]), _i32(t["pml_cell_param"])
        _check(lib.tlm_gpu_set_pml(self.h, int(t["n_pml_params"]), _p(pp), int(t["n_pml_cells"]), _p(pc)))
        if int(t.get("n_pml_material_cells", 0)):
            sg = _f64(t["pml_sigma"])
            _check(lib.tlm_gpu_set_pml_sigma(self.h, int(t["n_pml_params"]), _p(sg)))
        v, vf = _f64(t["fn_value"]), _f64(t["fn_value_face"])
        pts = [_i32(t[k]) for k in ("pt_cell", "pt_comp", "pt_fn", "pt_type")]
        _check(lib.tlm_gpu_set_excitation(self.h, int(t["n_functions"]), int(t["n_timesteps"]), _p(v), _p(vf),
                                          int(t["n_exc_points"]), *[_p(x) for x in pts], int(t["n_exc_cells"])))
        fa = [_i32(t[k]) for k in ("face_cx", "face_cy", "face_cz", "face_dir", "face_exc", "face_out")]
        _check(lib.tlm_gpu_set_faces(self.h, int(t["n_faces"]), *[_p(x) for x in fa], int(t["n_exc_faces"]),
                                     int(t["n_out_faces"])))
        fm = t.get("face_mat")
        if fm is not None and np.any(np.asarray(fm) != 0):
            fmv = _i32(fm)
            _check(lib.tlm_gpu_set_face_materials(self.h, int(t["n_faces"]), _p(fmv)))
        if np.any(np.asarray(t.get("wrap", (0, 0, 0))) != 0):
            w = [int(v) for v in t["wrap"]]
            _check(lib.tlm_gpu_set_wrap(self.h, w[0], w[1], w[2]))
        if int(t.get("n_smat", 0)):
            sf, sa, sb, so = _f64(t["smat_f"]), _f64(t["smat_a"]), _f64(t["smat_b"]), _i32(t["smat_order"])
            _check(lib.tlm_gpu_set_thin_layers(self.h, int(t["n_smat"]), _p(sf), _p(sa), _p(sb), _p(so),
                                               int(np.asarray(t["smat_a"]).shape[-1])))
            fs = _i32(t["face_smat"])
            _check(lib.tlm_gpu_set_face_thin_layers(self.h, int(t["n_faces"]), _p(fs)))
        if int(t["hs_n"]) and int(t.get("hs_outer", 0)):
            hc, ho, Ei, Hi = _i32(t["hs_cell"]), _f64(t["hs_offset"]), _f64(t["hs_Ei"]), _f64(t["hs_Hi"])
            _check(lib.tlm_gpu_set_outer_huygens(self.h, int(t["hs_n"]), _p(hc), _p(ho), _p(Ei), _p(Hi),
                                                 float(t["hs_offset_min"]), float(t["hs_c"]), int(t["hs_fn"])))
        elif int(t["hs_n"]):
            hf, hn, ho, Ei, Hi = (_i32(t["hs_face_exc"]), _i32(t["hs_norm"]), _f64(t["hs_offset"]), _f64(t["hs_Ei"]),
                                  _f64(t["hs_Hi"]))
            _check(lib.tlm_gpu_set_huygens(self.h, int(t["hs_n"]), _p(hf), _p(hn), _p(ho), _p(Ei), _p(Hi),
                                           float(t["hs_offset_min"]), float(t["hs_c"]), int(t["hs_fn"])))
        _check(lib.tlm_gpu_set_outputs(self.h, int(t["n_out_cells"])))
        keep = t.get("out_keep")
        if keep is not None and int(t["n_out_cells"]) and not np.all(np.asarray(keep) == 1):
            kp = _i32(keep)
            _check(lib.tlm_gpu_set_output_series(self.h, int(t["n_out_cells"]), _p(kp)))
        if int(t.get("n_vdft", 0)):
            vd = [_f64(t["vdft_freq"]), _i32(t["vdft_comp"]), _i32(t["vdft_first"]), _i32(t["vdft_last"]),
                  _i32(t["vdft_interval"]), _i32(t["vdft_cell_ptr"]), _i32(t["vdft_cell_out"])]
            _check(lib.tlm_gpu_set_volume_dft(self.h, int(t["n_vdft"]), *[_p(x) for x in vd]))
        if int(t.get("n_ps", 0)):
            pv = [_f64(t["ps_freq"]), _i32(t["ps_face_ptr"]), _i32(t["ps_face_out"]), _i32(t["ps_face_code"])]
            _check(lib.tlm_gpu_set_power_surfaces(self.h, int(t["n_ps"]), *[_p(x) for x in pv]))
        if int(t.get("n_modes", 0)):
            mv = [_i32(t["mode_comp"]), _i32(t["mode_face_ptr"]), _i32(t["mode_face_out"]), _i32(t["mode_face_code"]),
                  _f64(t["mode_field"])]
            _check(lib.tlm_gpu_set_mode_outputs(self.h, int(t["n_modes"]), *[_p(x) for x in mv]))
        if int(t.get("n_sar", 0)):
            sv = [_f64(t["sar_freq"]), _i32(t["sar_cell_ptr"]), _i32(t["sar_cell_out"])]
            _check(lib.tlm_gpu_set_sar_volumes(self.h, int(t["n_sar"]), *[_p(x) for x in sv]))
        if int(t.get("n_ovol", 0)):
            ov = [_i32(t[k]) for k in ("ovol_kind", "ovol_comp", "ovol_first", "ovol_last", "ovol_interval",
                                       "ovol_cell_ptr", "ovol_cell_out")]
            _check(lib.tlm_gpu_set_output_volumes(self.h, int(t["n_ovol"]), *[_p(x) for x in ov]))
        if int(t.get("rcs_on", 0)):
            rf, rc_, rd = _i32(t["rcs_face_out"]), _i32(t["rcs_face_code"]), _f64(t["rcs_face_dist"])
            _check(lib.tlm_gpu_set_rcs(self.h, float(t["rcs_theta"]), float(t["rcs_phi"]), int(t["rcs_npc"]),
                                       int(t["rcs_points"]), int(t["rcs_offset"]), len(rf), _p(rf), _p(rc_), _p(rd)))
        if int(t.get("n_osurf", 0)):
            os_ = [_i32(t[k]) for k in ("osurf_comp", "osurf_first", "osurf_last", "osurf_interval", "osurf_both",
                                        "osurf_face_ptr", "osurf_face_out", "osurf_face_code")]
            _check(lib.tlm_gpu_set_output_surfaces(self.h, int(t["n_osurf"]), *[_p(x) for x in os_]))
        if int(t["n_dft"]):
            df = [_f64(t["dft_freq"]), _i32(t["dft_comp"]), _i32(t["dft_face_ptr"]), _i32(t["dft_face_out"]),
                  _i32(t["dft_face_side"])]
            _check(lib.tlm_gpu_set_dft(self.h, int(t["n_dft"]), *[_p(x) for x in df]))
            if "dft_first" in t:
                dg = [_i32(t["dft_first"]), _i32(t["dft_last"]), _i32(t["dft_interval"])]
                _check(lib.tlm_gpu_set_dft_gate(self.h, int(t["n_dft"]), *[_p(x) for x in dg]))
        if int(t.get("n_ff", 0)):
            ff = [_f64(t["ff_freq"]), _i32(t["ff_face_ptr"]), _i32(t["ff_face_out"]), _i32(t["ff_face_code"])]
            _check(lib.tlm_gpu_set_far_field(self.h, int(t["n_ff"]), *[_p(x) for x in ff]))
        if int(t.get("n_face_points", 0)):
            fp = [_i32(t[k]) for k in ("fpt_face", "fpt_comp", "fpt_fn", "fpt_type")]
            _check(lib.tlm_gpu_set_face_excitation(self.h, int(t["n_face_points"]), *[_p(x) for x in fp]))
            if "fpt_side" in t and np.any(np.asarray(t["fpt_side"]) != 0):
                sd = _i32(t["fpt_side"])
                _check(lib.tlm_gpu_set_face_excitation_side(self.h, int(t["n_face_points"]), _p(sd)))
            if "fpt_scale" in t and np.any(np.asarray(t["fpt_scale"]) != 1.0):
                sc = _f64(t["fpt_scale"])
                _check(lib.tlm_gpu_set_face_excitation_scale(self.h, int(t["n_face_points"]), _p(sc)))
        if int(t.get("n_face_probes", 0)):
            fq = [_i32(t[k]) for k in ("fprobe_face", "fprobe_side", "fprobe_comp")]
            _check(lib.tlm_gpu_set_face_outputs(self.h, int(t["n_face_probes"]), *[_p(x) for x in fq]))
        if int(t.get("n_small_to_zero", 0)):
            _check(lib.tlm_gpu_set_small_to_zero(self.h, int(t["n_small_to_zero"]), float(t["small_to_zero_value"])))

    # -- time stepping -----------------------------------------------------
    def prepare(self):
        """Build the device state now rather than at the first run."""
        _check(_lib.tlm_gpu_prepare(self.h))

    def run(self, n_steps: int, sync: bool = True):
        _check(_lib.tlm_gpu_run(self.h, self.step + 1, n_steps))
        self.step += n_steps
        if sync:
            self.synchronize()

    def synchronize(self):
        _check(_lib.tlm_gpu_synchronize(self.h))

    def set_timing(self, enable: bool):
        _check(_lib.tlm_gpu_set_timing(self.h, 1 if enable else 0))

    def set_variant(self, variant: int):
        _check(_lib.tlm_gpu_set_variant(self.h, variant))

    def set_stream(self, stream_ptr: int):
        _check(_lib.tlm_gpu_set_stream(self.h, C.c_void_p(stream_ptr)))

    def last_run_time(self):
        a, b = C.c_float(0), C.c_float(0)
        _check(_lib.tlm_gpu_last_run_time(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def last_run_launches(self) -> int:
        n = C.c_int64(0)
        _check(_lib.tlm_gpu_last_run_launches(self.h, C.byref(n)))
        return n.value

    def memory_bytes(self) -> int:
        n = C.c_int64(0)
        _check(_lib.tlm_gpu_memory_bytes(self.h, C.byref(n)))
        return n.value

    # -- results -----------------------------------------------------------
    def cell_output(self, first: int = 1, n: Optional[int] = None) -> np.ndarray:
        """cell_output_field snapshots [n, n_kept, 6] of steps first.., for
        the output cells that keep a time series (all of them unless the
        tables' ``out_keep`` says otherwise), in output-number order."""
        if n is None:
            n = self.step - first + 1
        keep = self.t.get("out_keep")
        no = int(self.t["n_out_cells"]) if keep is None else int(np.sum(keep))
        out = np.zeros((n, max(no, 1), 6))
        _check(_lib.tlm_gpu_fetch_cell_output(self.h, first, n, out.ctypes.data_as(_f64p)))
        return out[:, :no, :]

    def face_output(self, first: int = 1, n: Optional[int] = None) -> np.ndarray:
        """Face output point series [n_face_probes, n] of steps first.."""
        if n is None:
            n = self.step - first + 1
        nq = int(self.t.get("n_face_probes", 0))
        out = np.zeros((max(n, 1), max(nq, 1)))
        _check(_lib.tlm_gpu_fetch_face_output(self.h, first, n, out.ctypes.data_as(_f64p)))
        return out[:n, :nq].T.copy()

    def far_field(self) -> np.ndarray:
        """Far-field accumulators [entries, 6] complex: Jx, Jy, Jz, Mx, My, Mz."""
        n = int(self.t["ff_face_ptr"][-1]) if int(self.t.get("n_ff", 0)) else 0
        out = np.zeros(max(12 * n, 12))
        _check(_lib.tlm_gpu_fetch_far_field(self.h, out.ctypes.data_as(_f64p)))
        v = out[: 12 * n].reshape(n, 6, 2)
        return v[..., 0] + 1j * v[..., 1]

    def power_surfaces(self) -> np.ndarray:
        """Power surface accumulators [entries, 4] complex: E1, E2, H1, H2 per face."""
        n = int(self.t["ps_face_ptr"][-1]) if int(self.t.get("n_ps", 0)) else 0
        out = np.zeros(max(8 * n, 8))
        _check(_lib.tlm_gpu_fetch_power_surfaces(self.h, out.ctypes.data_as(_f64p)))
        v = out[: 8 * n].reshape(n, 4, 2)
        return v[..., 0] + 1j * v[..., 1]

    def mode_outputs(self, first: int = 1, n: Optional[int] = None) -> np.ndarray:
        """Mode output values [n_modes, n] of steps first.."""
        if n is None:
            n = self.step - first + 1
        nm = int(self.t.get("n_modes", 0))
        out = np.zeros((max(n, 1), max(nm, 1)))
        _check(_lib.tlm_gpu_fetch_mode_outputs(self.h, first, n, out.ctypes.data_as(_f64p)))
        return out[:n, :nm].T.copy()

    def sar_volumes(self) -> np.ndarray:
        """SAR volume accumulators [entries, 3] complex: Ex, Ey, Ez per cell."""
        n = int(self.t["sar_cell_ptr"][-1]) if int(self.t.get("n_sar", 0)) else 0
        out = np.zeros(max(6 * n, 6))
        _check(_lib.tlm_gpu_fetch_sar_volumes(self.h, out.ctypes.data_as(_f64p)))
        v = out[: 6 * n].reshape(n, 3, 2)
        return v[..., 0] + 1j * v[..., 1]

    def output_volumes(self) -> list:
        """Time-domain output volume values, one array per volume: [n_output_steps,
        n_cells] for a "field" volume, [n_output_steps] for an average or a peak."""
        t = self.t
        shapes = []
        ptr = t.get("ovol_cell_ptr", [0])
        for k in range(int(t.get("n_ovol", 0))):
            first, last, every = int(t["ovol_first"][k]), int(t["ovol_last"][k]), int(t["ovol_interval"][k])
            hi = min(last, int(t["n_timesteps"]))
            ns = (hi - first) // every + 1 if hi >= first else 0
            shapes.append((ns, int(ptr[k + 1] - ptr[k])) if int(t["ovol_kind"][k]) == 0 else (ns,))
        total = sum(int(np.prod(s)) for s in shapes)
        out = np.zeros(max(total, 1))
        _check(_lib.tlm_gpu_fetch_output_volumes(self.h, out.ctypes.data_as(_f64p)))
        res, off = [], 0
        for s in shapes:
            n = int(np.prod(s))
            res.append(out[off:off + n].reshape(s).copy())
            off += n
        return res

    def rcs(self) -> np.ndarray:
        """RCS far-field arrays [4, n_points]: Etheta, Ephi, Htheta, Hphi."""
        n = int(self.t["rcs_points"]) if int(self.t.get("rcs_on", 0)) else 0
        out = np.zeros(max(4 * n, 4))
        _check(_lib.tlm_gpu_fetch_rcs(self.h, out.ctypes.data_as(_f64p)))
        return out[: 4 * n].reshape(4, n)

    def output_surfaces(self) -> list:
        """Time-domain output surface values: one array [n_output_steps,
        n_faces] per surface (rows of steps not run yet are zero)."""
        t = self.t
        shapes = output_surface_shapes(t)
        total = sum(a * b for a, b in shapes)
        out = np.zeros(max(total, 1))
        _check(_lib.tlm_gpu_fetch_output_surfaces(self.h, out.ctypes.data_as(_f64p)))
        res, off = [], 0
        for a, b in shapes:
            res.append(out[off:off + a * b].reshape(a, b).copy())
            off += a * b
        return res

    def volume_dft(self) -> np.ndarray:
        """Frequency output volume values [entries] complex, in the tables'
        volume then cell order."""
        n = int(self.t["vdft_cell_ptr"][-1]) if int(self.t.get("n_vdft", 0)) else 0
        out = np.zeros(max(2 * n, 2))
        _check(_lib.tlm_gpu_fetch_volume_dft(self.h, out.ctypes.data_as(_f64p)))
        v = out[: 2 * n].reshape(-1, 2)
        return v[:, 0] + 1j * v[:, 1]

    def dft(self) -> np.ndarray:
        n = int(self.t["dft_face_ptr"][-1]) if int(self.t["n_dft"]) else 0
        out = np.zeros(max(2 * n, 2))
        _check(_lib.tlm_gpu_fetch_dft(self.h, out.ctypes.data_as(_f64p)))
        return out[: 2 * n].reshape(-1, 2)

    def links(self) -> np.ndarray:
        t = self.t
        out = np.zeros(t["nx"] * t["ny"] * t["nz"] * 12)
        _check(_lib.tlm_gpu_fetch_links(self.h, out.ctypes.data_as(_f64p)))
        return out.reshape(t["nz"], t["ny"], t["nx"], 12)

    def halo_bytes(self) -> int:
        """Bytes of one side of the z-slab halo (two ports of a padded z-plane)."""
        v = C.c_int64(0)
        _check(_lib.tlm_gpu_halo_bytes(self.h, C.byref(v)))
        return int(v.value)

    def halo_get(self, side: int, dev_ptr: int):
        """Copy this slab's first (side 0) or last (side 1) plane's outgoing
        z pulses into device memory at ``dev_ptr``."""
        _check(_lib.tlm_gpu_halo_get(self.h, side, C.c_void_p(dev_ptr)))

    def halo_put(self, side: int, dev_ptr: int):
        """Fill the ghost plane below (side 0) or above (side 1) from device
        memory at ``dev_ptr`` (a neighbour slab's ``halo_get``)."""
        _check(_lib.tlm_gpu_halo_put(self.h, side, C.c_void_p(dev_ptr)))

    def close(self):
        if getattr(self, "h", 0):
            _check(_lib.tlm_gpu_destroy(self.h))
            self.h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class GpuBatch:
    """Several GpuMesh objects advanced together (one launch per kernel type
    per step, graph-replayed).  The meshes keep their own results."""

    def __init__(self, meshes):
        lib = load_library()
        self.meshes = list(meshes)
        arr = (C.c_int64 * len(self.meshes))(*[m.h for m in self.meshes])
        h = C.c_int64(0)
        _check(lib.tlm_gpu_batch_create(arr, len(self.meshes), C.byref(h)))
        self.h = h.value

    def set_variant(self, v: int):
        _check(_lib.tlm_gpu_batch_set_variant(self.h, v))

    def set_members(self, meshes):
        """Replace the batch's meshes (waits for its queued steps; the
        leavers can then be used alone or closed)."""
        meshes = list(meshes)
        arr = (C.c_int64 * len(meshes))(*[m.h for m in meshes])
        _check(_lib.tlm_gpu_batch_set_members(self.h, arr, len(meshes)))
        self.meshes = meshes

    def run(self, n_steps: int, sync: bool = True):
        _check(_lib.tlm_gpu_batch_run(self.h, n_steps))
        before = {id(m): m.step for m in self.meshes}
        for m in self.meshes:
            m.step = min(m.t["n_timesteps"], before[id(m)] + n_steps)
        if sync:
            self.synchronize()

    def synchronize(self):
        _check(_lib.tlm_gpu_batch_synchronize(self.h))

    def last_run(self):
        ms, cu, la = C.c_float(0), C.c_int64(0), C.c_int64(0)
        _check(_lib.tlm_gpu_batch_last_run(self.h, C.byref(ms), C.byref(cu), C.byref(la)))
        return ms.value, cu.value, la.value

    def close(self):
        if getattr(self, "h", 0):
            _check(_lib.tlm_gpu_batch_destroy(self.h))
            self.h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
