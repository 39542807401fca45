"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module, as the checker.  It runs the plain-C FP64 restatement of
GGI_TLM's sequential time loop (oracle/tlm_oracle.c) on the same tables the
GPU path consumes (ggi_tlm_b200.problem.build_tables).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtlm_oracle.so")
MAX_ORDER = 8

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)


class _Problem(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("n_timesteps", C.c_int32),
        ("dl", C.c_double), ("dt", C.c_double), ("R", C.c_double * 6),
        ("cell_code", _i32p), ("n_special", C.c_int32),
        ("sp_material", _i32p), ("sp_pml", _i32p), ("sp_excitation", _i32p), ("sp_output", _i32p),
        ("n_materials", C.c_int32), ("mat_type", _i32p), ("mat_eps_exists", _i32p), ("mat_mu_exists", _i32p),
        ("mat_eps_order", _i32p), ("mat_mu_order", _i32p),
        ("mat_Ys_eps_f", _f64p), ("mat_Zs_mu_f", _f64p), ("mat_Ge", _f64p), ("mat_Rm", _f64p),
        ("mat_eps_a", _f64p), ("mat_eps_b", _f64p), ("mat_mu_a", _f64p), ("mat_mu_b", _f64p),
        ("n_pml_params", C.c_int32), ("pml_params", _f64p), ("n_pml_cells", C.c_int32), ("pml_cell_param", _i32p),
        ("n_functions", C.c_int32), ("fn_value", _f64p), ("fn_value_face", _f64p),
        ("n_exc_points", C.c_int32), ("pt_cell", _i32p), ("pt_comp", _i32p), ("pt_fn", _i32p), ("pt_type", _i32p),
        ("n_exc_cells", C.c_int32),
        ("n_faces", C.c_int32), ("face_cx", _i32p), ("face_cy", _i32p), ("face_cz", _i32p), ("face_dir", _i32p),
        ("face_exc", _i32p), ("face_out", _i32p), ("n_exc_faces", C.c_int32), ("n_out_faces", C.c_int32),
        ("hs_n", C.c_int32), ("hs_face_exc", _i32p), ("hs_norm", _i32p), ("hs_offset", _f64p),
        ("hs_Ei", C.c_double * 3), ("hs_Hi", C.c_double * 3), ("hs_offset_min", C.c_double), ("hs_c", C.c_double),
        ("hs_fn", C.c_int32),
        ("n_out_cells", C.c_int32),
        ("n_dft", C.c_int32), ("dft_freq", _f64p), ("dft_comp", _i32p), ("dft_face_ptr", _i32p),
        ("dft_face_out", _i32p), ("dft_face_side", _i32p),
        ("n_small_to_zero", C.c_int32), ("small_to_zero_value", C.c_double),
        ("pml_sigma", _f64p),
        ("n_face_points", C.c_int32), ("fpt_face", _i32p), ("fpt_comp", _i32p), ("fpt_fn", _i32p),
        ("fpt_type", _i32p),
        ("n_face_probes", C.c_int32), ("fprobe_face", _i32p), ("fprobe_side", _i32p), ("fprobe_comp", _i32p),
        ("hs_outer", C.c_int32), ("hs_cell", _i32p),
        ("n_ff", C.c_int32), ("ff_freq", _f64p), ("ff_face_ptr", _i32p), ("ff_face_out", _i32p),
        ("ff_face_code", _i32p), ("face_mat", _i32p),
        ("face_smat", _i32p), ("n_smat", C.c_int32), ("smat_f", _f64p), ("smat_a", _f64p), ("smat_b", _f64p),
        ("smat_order", _i32p), ("wrap", C.c_int32 * 3), ("slab", C.c_int32 * 2),
        ("dft_gate", _i32p), ("fpt_side", _i32p), ("fpt_scale", _f64p),
    ]


def build(force: bool = False) -> str:
    """Compile oracle/_build/libtlm_oracle.so with the committed Makefile."""
    src = os.path.join(_HERE, "tlm_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB_PATH


_lib = None


def _load():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.tlm_oracle_create.restype = C.c_void_p
        _lib.tlm_oracle_create.argtypes = [C.POINTER(_Problem)]
        _lib.tlm_oracle_destroy.argtypes = [C.c_void_p]
        _lib.tlm_oracle_run.argtypes = [C.c_void_p, C.c_int32, C.c_int32, _f64p]
        _lib.tlm_oracle_get_dft.argtypes = [C.c_void_p, _f64p]
        _lib.tlm_oracle_get_links.argtypes = [C.c_void_p, _f64p]
        _lib.tlm_oracle_get_face_probes.argtypes = [C.c_void_p, _f64p]
        _lib.tlm_oracle_get_far_field.argtypes = [C.c_void_p, _f64p]
        _lib.tlm_oracle_set_threads.argtypes = [C.c_void_p, C.c_int32]
        _lib.tlm_oracle_set_threads.restype = C.c_int32
        _lib.tlm_oracle_half_step.argtypes = [C.c_void_p, C.c_int32, C.c_int32, _f64p]
        _lib.tlm_oracle_get_zplane.argtypes = [C.c_void_p, C.c_int32, _f64p]
        _lib.tlm_oracle_set_zplane.argtypes = [C.c_void_p, C.c_int32, _f64p]
    return _lib


class Oracle:
    """One oracle instance over one problem's tables."""

    def __init__(self, t: dict, threads: int = 1):
        lib = _load()
        self.t = t
        keep = []

        def arr_empty():
            a = np.zeros(1, dtype=np.int32)
            keep.append(a)
            return a.ctypes.data_as(_i32p)

        def arr_empty_f():
            a = np.zeros(1)
            keep.append(a)
            return a.ctypes.data_as(_f64p)

        def arr(key, dtype):
            a = np.ascontiguousarray(t[key], dtype=dtype).reshape(-1)
            if a.size == 0:
                a = np.zeros(1, dtype=dtype)
            keep.append(a)
            return a.ctypes.data_as(_i32p if dtype == np.int32 else _f64p)

        p = _Problem()
        p.nx, p.ny, p.nz, p.n_timesteps = t["nx"], t["ny"], t["nz"], t["n_timesteps"]
        p.dl, p.dt = t["dl"], t["dt"]
        p.R[:] = [float(v) for v in t["R"]]
        p.cell_code = arr("cell_code", np.int32)
        p.n_special = t["n_special"]
        for k in ("sp_material", "sp_pml", "sp_excitation", "sp_output", "mat_type", "mat_eps_exists",
                  "mat_mu_exists", "mat_eps_order", "mat_mu_order", "pml_cell_param", "pt_cell", "pt_comp",
                  "pt_fn", "pt_type", "face_cx", "face_cy", "face_cz", "face_dir", "face_exc", "face_out",
                  "hs_face_exc", "hs_norm", "dft_comp", "dft_face_ptr", "dft_face_out", "dft_face_side"):
            setattr(p, k, arr(k, np.int32))
        for k in ("mat_Ys_eps_f", "mat_Zs_mu_f", "mat_Ge", "mat_Rm", "mat_eps_a", "mat_eps_b", "mat_mu_a",
                  "mat_mu_b", "pml_params", "fn_value", "fn_value_face", "hs_offset", "dft_freq"):
            setattr(p, k, arr(k, np.float64))
        for k in ("n_materials", "n_pml_params", "n_pml_cells", "n_functions", "n_exc_points", "n_exc_cells",
                  "n_faces", "n_exc_faces", "n_out_faces", "hs_n", "hs_fn", "n_out_cells", "n_dft"):
            setattr(p, k, int(t[k]))
        p.hs_Ei[:] = [float(v) for v in t["hs_Ei"]]
        p.hs_Hi[:] = [float(v) for v in t["hs_Hi"]]
        p.hs_offset_min = float(t["hs_offset_min"])
        p.hs_c = float(t["hs_c"])
        p.n_face_points = int(t.get("n_face_points", 0))
        p.n_face_probes = int(t.get("n_face_probes", 0))
        p.hs_outer = int(t.get("hs_outer", 0))
        p.n_ff = int(t.get("n_ff", 0))
        p.ff_freq = arr("ff_freq", np.float64) if "ff_freq" in t else arr_empty_f()
        for k in ("ff_face_ptr", "ff_face_out", "ff_face_code"):
            setattr(p, k, arr(k, np.int32) if k in t else arr_empty())
        if "face_mat" in t and np.any(np.asarray(t["face_mat"]) != 0):
            p.face_mat = arr("face_mat", np.int32)  # else NULL: no surface materials
        p.wrap[:] = [int(v) for v in t.get("wrap", (0, 0, 0))]
        p.slab[:] = [int(v) for v in t.get("slab", (0, 0))]
        if int(t.get("n_dft", 0)) and "dft_first" in t:
            g = np.ascontiguousarray(np.stack([t["dft_first"], t["dft_last"], t["dft_interval"]], axis=1),
                                     dtype=np.int32)
            keep.append(g)
            p.dft_gate = g.ctypes.data_as(_i32p)
        if int(t.get("n_smat", 0)):
            p.face_smat = arr("face_smat", np.int32)
            p.n_smat = int(t["n_smat"])
            for k in ("smat_f", "smat_a", "smat_b"):
                setattr(p, k, arr(k, np.float64))
            p.smat_order = arr("smat_order", np.int32)
        for k in ("fpt_face", "fpt_comp", "fpt_fn", "fpt_type", "fpt_side", "fprobe_face", "fprobe_side",
                  "fprobe_comp", "hs_cell"):
            setattr(p, k, arr(k, np.int32) if k in t else arr_empty())
        if "fpt_scale" in t and int(t.get("n_face_points", 0)):
            p.fpt_scale = arr("fpt_scale", np.float64)
        if int(t.get("n_pml_material_cells", 0)):
            p.pml_sigma = arr("pml_sigma", np.float64)
        p.n_small_to_zero = int(t.get("n_small_to_zero", 0))
        p.small_to_zero_value = float(t.get("small_to_zero_value", 0.0))
        self._keep = keep
        self._p = p
        self._h = lib.tlm_oracle_create(C.byref(p))
        if not self._h:
            raise MemoryError("oracle allocation failed")
        self.threads = lib.tlm_oracle_set_threads(self._h, int(threads))
        self.step = 0

    def run(self, n_steps: int) -> np.ndarray:
        """Advance n_steps; returns cell_output_field snapshots [n, n_out_cells, 6]."""
        n_out = max(int(self.t["n_out_cells"]), 1)
        out = np.zeros((n_steps, n_out, 6))
        rc = _load().tlm_oracle_run(self._h, self.step + 1, n_steps, out.ctypes.data_as(_f64p))
        if rc != 0:
            raise RuntimeError(f"oracle run failed rc={rc}")
        self.step += n_steps
        return out[:, : int(self.t["n_out_cells"]), :]

    def half_step(self, half: int) -> np.ndarray:
        """Half 1 (excitation, scatter, cell output: returns that step's
        cell_output_field [n_out_cells, 6]) or half 2 (connect to the outer
        boundary) of the next timestep, for a partitioned run that exchanges
        z-planes between the halves (TLM_parallel_pass_data_1/2)."""
        ts = self.step + 1
        out = np.zeros((max(int(self.t["n_out_cells"]), 1), 6))
        rc = _load().tlm_oracle_half_step(self._h, ts, half, out.ctypes.data_as(_f64p))
        if rc != 0:
            raise RuntimeError(f"oracle half step failed rc={rc}")
        if half == 2:
            self.step = ts
        return out[: int(self.t["n_out_cells"])]

    def zplane(self, plane: int) -> np.ndarray:
        """Vx_zmax, Vy_zmax of the ghost plane below the slab (0) or of its
        top plane (1), as [2, ny, nx]."""
        out = np.zeros((2, int(self.t["ny"]), int(self.t["nx"])))
        _load().tlm_oracle_get_zplane(self._h, plane, out.ctypes.data_as(_f64p))
        return out

    def set_zplane(self, plane: int, v: np.ndarray):
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(2, int(self.t["ny"]), int(self.t["nx"]))
        _load().tlm_oracle_set_zplane(self._h, plane, v.ctypes.data_as(_f64p))

    def dft(self) -> np.ndarray:
        n = int(self.t["dft_face_ptr"][-1]) if self.t["n_dft"] else 0
        out = np.zeros(max(2 * n, 1))
        _load().tlm_oracle_get_dft(self._h, out.ctypes.data_as(_f64p))
        return out[: 2 * n].reshape(-1, 2)

    def far_field(self) -> np.ndarray:
        """Far-field accumulators [entries, 6] complex: Jx, Jy, Jz, Mx, My, Mz."""
        n = int(self.t["ff_face_ptr"][-1]) if int(self.t.get("n_ff", 0)) else 0
        out = np.zeros(max(12 * n, 1))
        _load().tlm_oracle_get_far_field(self._h, out.ctypes.data_as(_f64p))
        v = out[: 12 * n].reshape(n, 6, 2)
        return v[..., 0] + 1j * v[..., 1]

    def face_probes(self) -> np.ndarray:
        """Face output point values [n_face_probes, steps run so far]."""
        n = int(self.t.get("n_face_probes", 0))
        out = np.zeros(max(self.step * n, 1))
        _load().tlm_oracle_get_face_probes(self._h, out.ctypes.data_as(_f64p))
        return out[: self.step * n].reshape(self.step, n).T.copy()

    def links(self) -> np.ndarray:
        t = self.t
        out = np.zeros(t["nx"] * t["ny"] * t["nz"] * 12)
        _load().tlm_oracle_get_links(self._h, out.ctypes.data_as(_f64p))
        return out.reshape(t["nz"], t["ny"], t["nx"], 12)

    def close(self):
        if self._h:
            _load().tlm_oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def volume_dft(t: dict, cell_out: np.ndarray) -> np.ndarray:
    """Frequency output volumes, restating cell_output_frequency_output_volumes
    (OUTPUT/frequency_output_volumes.F90:309-390) over the oracle's
    cell_output_field history cell_out [steps, n_out_cells, 6] (from
    ``Oracle.run``): on every step that get_output_flag (OUTPUT/output.F90:
    564-598) accepts, value(cell) = value(cell) + field * exp(-j*2*pi*f*time)
    with time = (timestep-1)*dt (TLM_SOLVER/run_TLM.F90:240-243, before the
    half step).  Returns the values [entries] in volume then cell order."""
    n = int(t.get("n_vdft", 0))
    ptr = t["vdft_cell_ptr"]
    out = []
    for v in range(n):
        cells = np.asarray(t["vdft_cell_out"][ptr[v]:ptr[v + 1]], dtype=np.int64) - 1
        comp = int(t["vdft_comp"][v]) - 1
        first, last, every = int(t["vdft_first"][v]), int(t["vdft_last"][v]), int(t["vdft_interval"][v])
        f = float(t["vdft_freq"][v])
        acc = np.zeros(len(cells), dtype=np.complex128)
        for timestep in range(1, cell_out.shape[0] + 1):
            if timestep < first or timestep > last or (timestep - first) % every != 0:
                continue
            time = (timestep - 1) * t["dt"]
            ejwt = np.exp(-1j * 2.0 * np.pi * f * time)
            acc = acc + cell_out[timestep - 1, cells, comp] * ejwt
        out.append(acc)
    return np.concatenate(out) if out else np.zeros(0, dtype=np.complex128)


def output_surfaces(t: dict) -> list:
    """Time-domain output surfaces, restating face_output_surfaces
    (OUTPUT/output_surfaces.F90:601-760) on the oracle's face fields: the
    oracle runs the whole solve with face output points added on both sides
    (1, 2) and all six components of every surface face, and each output
    step (get_output_flag, OUTPUT/output.F90:564-598) takes, per face,
    field = side of the face code (or side 1 and field2 = side 2 with both
    sides), the normal +1 on a min face and -1 on a max face, and the
    component: E/H, J = n x H(field) - n x H(field2), |E|, |H| or |J|.
    Returns one array [n_output_steps, n_faces] per surface."""
    ns = int(t.get("n_osurf", 0))
    if not ns:
        return []
    ptr = t["osurf_face_ptr"]
    fo = np.asarray(t["osurf_face_out"], dtype=np.int32)
    n0 = int(t.get("n_face_probes", 0))
    add_face = np.repeat(fo, 12)
    add_side = np.tile(np.repeat(np.array([1, 2], dtype=np.int32), 6), len(fo))
    add_comp = np.tile(np.arange(1, 7, dtype=np.int32), 2 * len(fo))
    t2 = dict(t)
    t2["n_face_probes"] = n0 + len(add_face)
    t2["fprobe_face"] = np.concatenate([np.asarray(t.get("fprobe_face", []), dtype=np.int32), add_face])
    t2["fprobe_side"] = np.concatenate([np.asarray(t.get("fprobe_side", []), dtype=np.int32), add_side])
    t2["fprobe_comp"] = np.concatenate([np.asarray(t.get("fprobe_comp", []), dtype=np.int32), add_comp])
    o = Oracle(t2)
    o.run(int(t["n_timesteps"]))
    vals = o.face_probes()[n0:].reshape(len(fo), 2, 6, -1)  # [face, side, comp, step]
    res = []
    for k in range(ns):
        faces = range(ptr[k], ptr[k + 1])
        comp, both = int(t["osurf_comp"][k]), bool(t["osurf_both"][k])
        first, last, every = int(t["osurf_first"][k]), int(t["osurf_last"][k]), int(t["osurf_interval"][k])
        steps = [s for s in range(first, min(last, int(t["n_timesteps"])) + 1) if (s - first) % every == 0]
        out = np.zeros((len(steps), len(faces)))
        for j, f in enumerate(faces):
            code = int(t["osurf_face_code"][f])
            side = 0 if code <= 3 else 1
            n = [0.0, 0.0, 0.0]
            n[(code - 1) % 3] = 1.0 if code <= 3 else -1.0
            normx, normy, normz = n
            for r, s in enumerate(steps):
                field = vals[f, 0 if both else side, :, s - 1]
                field2 = vals[f, 1, :, s - 1] if both else np.zeros(6)
                Ex, Ey, Ez, Hx, Hy, Hz = field
                Jsx = (normy * Hz - normz * Hy) - (normy * field2[5] - normz * field2[4])
                Jsy = (normz * Hx - normx * Hz) - (normz * field2[3] - normx * field2[5])
                Jsz = (normx * Hy - normy * Hx) - (normx * field2[4] - normy * field2[3])
                if comp <= 6:
                    v = field[comp - 1]
                elif comp in (7, 8, 9):
                    v = (Jsx, Jsy, Jsz)[comp - 7]
                elif comp == 13:
                    v = np.sqrt(Ex ** 2 + Ey ** 2 + Ez ** 2)
                elif comp == 14:
                    v = np.sqrt(Hx ** 2 + Hy ** 2 + Hz ** 2)
                else:
                    v = np.sqrt(Jsx ** 2 + Jsy ** 2 + Jsz ** 2)
                out[r, j] = v
        res.append(out)
    return res


def rcs(t: dict) -> np.ndarray:
    """The RCS surface's time-domain far field, restating face_output_rcs
    (OUTPUT/RCS_surfaces.F90:386-560) on the oracle's face fields: the oracle
    runs the whole solve with face output points added on each RCS face's
    side for all six components; every step, for every face in list order,
    point = INT(n_rcs_points_per_cell * (-(K.x) + time*c0) / dl) - offset
    with time = (timestep-1)*dt + dt/2, and when 1 <= point <= n_points the
    face adds Etheta, Ephi, Htheta, Hphi there.  Returns [4, n_points]."""
    if not int(t.get("rcs_on", 0)):
        return np.zeros((4, 0))
    fo = np.asarray(t["rcs_face_out"], dtype=np.int32)
    codes = np.asarray(t["rcs_face_code"], dtype=np.int32)
    sides = np.where(codes <= 3, 1, 2).astype(np.int32)
    n0 = int(t.get("n_face_probes", 0))
    t2 = dict(t)
    t2["n_face_probes"] = n0 + 6 * len(fo)
    t2["fprobe_face"] = np.concatenate([np.asarray(t.get("fprobe_face", []), dtype=np.int32), np.repeat(fo, 6)])
    t2["fprobe_side"] = np.concatenate([np.asarray(t.get("fprobe_side", []), dtype=np.int32), np.repeat(sides, 6)])
    t2["fprobe_comp"] = np.concatenate([np.asarray(t.get("fprobe_comp", []), dtype=np.int32),
                                        np.tile(np.arange(1, 7, dtype=np.int32), len(fo))])
    o = Oracle(t2)
    o.run(int(t["n_timesteps"]))
    vals = o.face_probes()[n0:].reshape(len(fo), 6, -1)  # [face, comp, step]
    theta, phi = float(t["rcs_theta"]), float(t["rcs_phi"])
    ct, st, cp, sp = math.cos(theta), math.sin(theta), math.cos(phi), math.sin(phi)
    dl, dt = float(t["dl"]), float(t["dt"])
    dA, four_pi = dl * dl, 4.0 * math.pi
    npc, n_pts, offset = int(t["rcs_npc"]), int(t["rcs_points"]), int(t["rcs_offset"])
    dist = np.asarray(t["rcs_face_dist"], dtype=np.float64)
    acc = np.zeros((4, n_pts))
    Z0 = 376.73031346177
    for timestep in range(1, int(t["n_timesteps"]) + 1):
        time = (timestep - 1) * dt
        time = time + dt / 2.0
        tc0 = time * 2.99792458e8
        for f in range(len(fo)):
            dm = -float(dist[f]) + tc0
            point = int(float(npc) * dm / dl) - offset
            if point < 1 or point > n_pts:
                continue
            code = int(codes[f])
            n = [0.0, 0.0, 0.0]
            n[(code - 1) % 3] = 1.0 if code <= 3 else -1.0
            normx, normy, normz = n
            Ex, Ey, Ez, Hx, Hy, Hz = (float(v) for v in vals[f, :, timestep - 1])
            Jsx, Jsy, Jsz = normy * Hz - normz * Hy, normz * Hx - normx * Hz, normx * Hy - normy * Hx
            Msx, Msy, Msz = -(normy * Ez - normz * Ey), -(normz * Ex - normx * Ez), -(normx * Ey - normy * Ex)
            Nt = (Jsx * ct * cp + Jsy * ct * sp - Jsz * st) * dA / four_pi
            Np = (-Jsx * sp + Jsy * cp) * dA / four_pi
            Lt = (Msx * ct * cp + Msy * ct * sp - Msz * st) * dA / four_pi
            Lp = (-Msx * sp + Msy * cp) * dA / four_pi
            acc[0, point - 1] += -(Lp + Z0 * Nt)
            acc[1, point - 1] += Lt - Z0 * Np
            acc[2, point - 1] += Np - Lt / Z0
            acc[3, point - 1] += -(Nt + Lp / Z0)
    return acc


def output_volumes(t: dict, cell_out: np.ndarray) -> list:
    """Time-domain output volumes over the oracle's cell_output_field history
    cell_out [steps, n_out_cells, 6], on every step get_output_flag accepts:
    kind 0 each cell's field (OUTPUT/output_volumes.F90 cell_output_volumes),
    kind 1 the sum in list order over the number of cells
    (output_volume_averages.F90), kind 2 the largest |field| starting from 0
    (output_volume_peak.F90); kinds 1 and 2 give 0 below 1e-30.  Returns one
    array per volume ([n_output_steps, n_cells] or [n_output_steps])."""
    res = []
    ptr = t.get("ovol_cell_ptr", [0])
    for k in range(int(t.get("n_ovol", 0))):
        cells = np.asarray(t["ovol_cell_out"][ptr[k]:ptr[k + 1]], dtype=np.int64) - 1
        comp, kind = int(t["ovol_comp"][k]) - 1, int(t["ovol_kind"][k])
        first, last, every = int(t["ovol_first"][k]), int(t["ovol_last"][k]), int(t["ovol_interval"][k])
        rows = []
        for timestep in range(first, min(last, cell_out.shape[0]) + 1):
            if (timestep - first) % every:
                continue
            f = cell_out[timestep - 1, cells, comp]
            if kind == 0:
                rows.append(f.copy())
                continue
            v = 0.0
            for x in f:
                v = v + float(x) if kind == 1 else max(v, abs(float(x)))
            if kind == 1:
                v = v / float(len(cells)) if len(cells) else 0.0
            rows.append(0.0 if abs(v) < 1e-30 else v)
        res.append(np.array(rows))
    return res


def sar_volumes(t: dict, cell_out: np.ndarray) -> np.ndarray:
    """SAR volume accumulators, restating cell_output_SAR_volumes
    (OUTPUT/SAR_volumes.F90:257-330) over the oracle's cell_output_field
    history: every step, E_c = E_c + ejwt * field_c * dt for c = x, y, z,
    ejwt = exp(-j*2*pi*f*time), time = (timestep-1)*dt.  Returns [entries, 3]."""
    n = int(t.get("n_sar", 0))
    ptr = t["sar_cell_ptr"] if n else [0]
    dt = float(t["dt"])
    out = []
    for v in range(n):
        cells = np.asarray(t["sar_cell_out"][ptr[v]:ptr[v + 1]], dtype=np.int64) - 1
        f = float(t["sar_freq"][v])
        acc = np.zeros((len(cells), 3), dtype=np.complex128)
        for timestep in range(1, cell_out.shape[0] + 1):
            time = (timestep - 1) * dt
            ejwt = np.exp(-1j * 2.0 * np.pi * f * time)
            acc = acc + ejwt * cell_out[timestep - 1][cells][:, 0:3] * dt
        out.append(acc)
    return np.concatenate(out) if out else np.zeros((0, 3), dtype=np.complex128)


def _face_field_probes(t: dict, fo, codes) -> np.ndarray:
    """Run the oracle over the whole solve with face output points on each
    listed face's side (face code 1..3 -> side 1, 4..6 -> side 2) for all six
    components; returns the values [face, component, step]."""
    fo = np.asarray(fo, dtype=np.int32)
    sides = np.where(np.asarray(codes) <= 3, 1, 2).astype(np.int32)
    n0 = int(t.get("n_face_probes", 0))
    t2 = dict(t)
    t2["n_face_probes"] = n0 + 6 * len(fo)
    t2["fprobe_face"] = np.concatenate([np.asarray(t.get("fprobe_face", []), dtype=np.int32), np.repeat(fo, 6)])
    t2["fprobe_side"] = np.concatenate([np.asarray(t.get("fprobe_side", []), dtype=np.int32), np.repeat(sides, 6)])
    t2["fprobe_comp"] = np.concatenate([np.asarray(t.get("fprobe_comp", []), dtype=np.int32),
                                        np.tile(np.arange(1, 7, dtype=np.int32), len(fo))])
    o = Oracle(t2)
    o.run(int(t["n_timesteps"]))
    return o.face_probes()[n0:].reshape(len(fo), 6, -1)


def power_surfaces(t: dict) -> np.ndarray:
    """Frequency-domain power surfaces, restating
    face_output_frequency_domain_power_surfaces
    (OUTPUT/frequency_domain_power_surfaces.F90:287-420): every step each face
    adds E1, E2, H1, H2 (tangential fields on its side) * exp(-j*2*pi*f*time),
    time = (timestep-1)*dt + dt/2.  Returns [entries, 4]."""
    n = int(t.get("n_ps", 0))
    if not n:
        return np.zeros((0, 4), dtype=np.complex128)
    vals = _face_field_probes(t, t["ps_face_out"], t["ps_face_code"])
    ptr, codes = t["ps_face_ptr"], np.asarray(t["ps_face_code"])
    pick = {0: (1, 2, 4, 5), 1: (2, 0, 5, 3), 2: (0, 1, 3, 4)}  # (E1, E2, H1, H2) by face axis
    acc = np.zeros((len(codes), 4), dtype=np.complex128)
    dt = float(t["dt"])
    for v in range(n):
        f = float(t["ps_freq"][v])
        for timestep in range(1, int(t["n_timesteps"]) + 1):
            time = (timestep - 1) * dt
            time = time + dt / 2.0
            ejwt = np.exp(-1j * 2.0 * np.pi * f * time)
            for k in range(ptr[v], ptr[v + 1]):
                comps = pick[(int(codes[k]) - 1) % 3]
                for c in range(4):
                    acc[k, c] = acc[k, c] + vals[k, comps[c], timestep - 1] * ejwt
    return acc


def mode_outputs(t: dict) -> np.ndarray:
    """Mode outputs, restating Mode_output (OUTPUT/output_modes.F90:546-620):
    every step the sum in list order of face_output_field(side, component) *
    mode_field over the mode's faces, 0 below 1e-30.  Returns [n_modes, steps]."""
    n = int(t.get("n_modes", 0))
    if not n:
        return np.zeros((0, int(t["n_timesteps"])))
    vals = _face_field_probes(t, t["mode_face_out"], t["mode_face_code"])
    ptr, w = t["mode_face_ptr"], np.asarray(t["mode_field"])
    out = np.zeros((n, int(t["n_timesteps"])))
    for v in range(n):
        comp = int(t["mode_comp"][v]) - 1
        for s in range(int(t["n_timesteps"])):
            acc = 0.0
            for k in range(ptr[v], ptr[v + 1]):
                acc = acc + float(vals[k, comp, s]) * float(w[k])
            out[v, s] = 0.0 if abs(acc) < 1e-30 else acc
    return out
