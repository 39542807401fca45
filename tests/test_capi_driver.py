"""The C ABI driven from C++ with no Python in the process (tests/capi_driver.cpp):
the call sequence a Fortran driver makes in place of run_TLM, from plain
arrays, running in chunks of 100 steps and reading the output points back
after each chunk.

CPU: the driver compiles and links against the library, and without a GPU
it stops with the library's error message and exit code 1, as the Fortran
shim does.  GPU: its results equal the Python binding's bit for bit, and in
FP64 the oracle's to 1e-10."""
import dataclasses
import os
import subprocess
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import build, capi, cases
from ggi_tlm_b200.problem import OutputPoint, PointExcitation, build_tables, probe_series

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import oracle  # noqa: E402

INTS = ["cell_code", "sp_material", "sp_pml", "sp_excitation", "sp_output", "mat_type", "mat_eps_exists",
        "mat_mu_exists", "mat_eps_order", "mat_mu_order", "pml_cell_param", "pt_cell", "pt_comp", "pt_fn", "pt_type",
        "face_cx", "face_cy", "face_cz", "face_dir", "face_exc", "face_out", "hs_face_exc", "hs_norm", "fpt_face",
        "fpt_comp", "fpt_fn", "fpt_type", "fprobe_face", "fprobe_side", "fprobe_comp", "dft_comp", "dft_face_ptr",
        "dft_face_out", "dft_face_side", "dft_first", "dft_last", "dft_interval"]
DOUBLES = ["R", "mat_Ys_eps_f", "mat_Zs_mu_f", "mat_Ge", "mat_Rm", "mat_eps_a", "mat_eps_b", "mat_mu_a", "mat_mu_b",
           "pml_params", "fn_value", "fn_value_face", "hs_offset", "hs_Ei", "hs_Hi", "dft_freq"]
SCALARS = ["nx", "ny", "nz", "n_timesteps", "dl", "dt", "n_special", "n_materials", "n_pml_params", "n_pml_cells",
           "n_functions", "n_exc_points", "n_exc_cells", "n_faces", "n_exc_faces", "n_out_faces", "hs_n",
           "hs_offset_min", "hs_c", "hs_fn", "n_out_cells", "n_face_points", "n_face_probes", "n_dft"]


def write_tables(t, d):
    """The tables in the driver's format: manifest.txt plus one raw file per array."""
    assert not int(t.get("hs_outer", 0)) and not int(t.get("n_vdft", 0)) and not int(t.get("n_pml_material_cells", 0))
    os.makedirs(d, exist_ok=True)
    lines = []
    for k in INTS + DOUBLES:
        a = np.asarray(t.get(k, []), dtype=np.int32 if k in INTS else np.float64).reshape(-1)
        a.tofile(os.path.join(d, k + ".bin"))
        lines.append(f"{k} {'i' if k in INTS else 'd'} {a.size}")
    nm = int(t["n_materials"])
    stride = np.asarray(t["mat_eps_a"]).reshape(nm, -1).shape[1] if nm else 1
    for k, v in [(k, t.get(k, 0)) for k in SCALARS] + [("mat_stride", stride), ("n_kept", t["n_out_cells"])]:
        lines.append(f"{k} s {float(v)!r}")
    with open(os.path.join(d, "manifest.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")


def compile_driver(tmp):
    exe = os.path.join(tmp, "capi_driver")
    lib_dir = os.path.dirname(build.LIB)
    cmd = ["g++", "-O1", "-std=c++17", "-o", exe, os.path.join(HERE, "capi_driver.cpp"), f"-L{lib_dir}", "-ltlm_gpu",
           f"-Wl,-rpath,{lib_dir}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


def specs():
    a = cases.pml_spheres(n=24, pml=4, n_spheres=3, steps=230, n_probes=4, n_freq=3, dft_size=6, rmin=2.0, rmax=3.5)
    a.dft_surfaces = [dataclasses.replace(d, first_step=20, last_step=200, interval=3) for d in a.dft_surfaces]
    b = cases.pml_point_source(18, pml=3, steps=150, n_probes=2)
    b.point_excitations.append(PointExcitation((9, 9, 6), "Ex", 1, face="zmin"))
    b.outputs.append(OutputPoint((9, 10, 11), "Hy", face="xmax"))
    return [a, b]


def run_driver(exe, t, tmp, precision):
    tdir, odir = os.path.join(tmp, "tables"), os.path.join(tmp, "out")
    write_tables(t, tdir)
    os.makedirs(odir, exist_ok=True)
    return subprocess.run([exe, tdir, odir, str(precision)], capture_output=True, text=True, timeout=600), odir


def test_driver_builds_and_stops_cleanly_without_a_gpu(tmp_path):
    import torch

    build.build()
    exe = compile_driver(str(tmp_path))
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU test runs the driver")
    res, _ = run_driver(exe, build_tables(specs()[1]), str(tmp_path), 64)
    assert res.returncode == 1
    assert "ERROR in run_TLM_gpu:" in res.stderr


@pytest.mark.gpu
def test_driver_matches_binding_and_oracle(gpu_lib, tmp_path):
    exe = compile_driver(str(tmp_path))
    for spec in specs():
        t = build_tables(spec)
        steps, no, nf = t["n_timesteps"], int(t["n_out_cells"]), int(t["n_face_probes"])
        for prec in (capi.TLM_PRECISION_FP64, capi.TLM_PRECISION_FP32):
            res, odir = run_driver(exe, t, str(tmp_path), prec)
            assert res.returncode == 0, res.stderr
            co = np.fromfile(os.path.join(odir, "cell_out.bin")).reshape(steps, no, 6)
            fo = np.fromfile(os.path.join(odir, "face_out.bin")).reshape(steps, nf).T
            dft = np.fromfile(os.path.join(odir, "dft.bin")).reshape(-1, 2)
            with capi.GpuMesh(t, precision=prec) as g:
                g.run(steps)
                assert np.array_equal(co, g.cell_output())
                assert np.array_equal(fo, g.face_output())
                if int(t["n_dft"]):
                    assert np.array_equal(dft, g.dft())
            if prec == capi.TLM_PRECISION_FP64:
                o = oracle.Oracle(t)
                want = probe_series(t, o.run(steps))
                for a, b in zip(probe_series(t, co), want):
                    assert np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(b)
                if nf:
                    fw = o.face_probes()
                    assert np.linalg.norm(fo - fw) <= 1e-10 * np.linalg.norm(fw)
