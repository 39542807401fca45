"""The problem-file runner (python -m ggi_tlm_b200.run): .inp in, .tout out.

CPU: the files it writes, from the oracle's results of the reference's
HUYGENS_SURFACE input, carry the reference's header and the golden centre
series; volume average and peak files follow their output steps and
numbering; without a GPU the runner stops with the library's message and
exit code 1.  GPU: the runner's own files against the oracle's."""
import os
import subprocess
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import run as runner
from ggi_tlm_b200.inp import read_inp
from ggi_tlm_b200.problem import build_tables
from ggi_tlm_b200.tout import read_tout

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "oracle"))
import oracle  # noqa: E402
import test_inp  # noqa: E402

TOL = 5e-7  # E16.7


def problem_dir(tmp, name, text):
    """A run directory holding <name>.inp and the material files it names."""
    with open(os.path.join(tmp, name + ".inp"), "w", encoding="latin-1") as f:
        f.write("\n".join(text) + "\n")
    os.makedirs(os.path.join(tmp, "MATERIAL_DIRECTORY"), exist_ok=True)
    d = np.load(os.path.join(HERE, "golden", "vmat_text.npz"))
    for k in d.files:
        with open(os.path.join(tmp, "MATERIAL_DIRECTORY", k + ".vmat"), "w") as f:
            f.write("\n".join(str(x) for x in d[k]) + "\n")
    return tmp


def oracle_files(tmp, name, lines):
    p = read_inp(lines, test_inp.materials)
    t = build_tables(p.spec)
    o = oracle.Oracle(t)
    cell = o.run(t["n_timesteps"])
    face = o.face_probes() if int(t["n_face_probes"]) else np.zeros((0, t["n_timesteps"]))
    vols = oracle.output_volumes(t, cell) if p.spec.output_volumes else None
    power = oracle.power_surfaces(t) if p.spec.power_surfaces else None
    surfs = oracle.output_surfaces(t) if p.spec.output_surfaces else None
    dft = o.dft() if p.spec.dft_surfaces else None
    far = o.far_field() if p.spec.far_field_surfaces else None
    rcs = oracle.rcs(t) if p.spec.rcs_surface is not None else None
    modes = oracle.mode_outputs(t) if p.spec.mode_outputs else None
    return runner.write_results(name, p, t, cell, face, vols, tmp, power, far, rcs=rcs, surfaces=surfs, dft=dft,
                                modes=modes), p, t


# ALL_OUTPUTS with an output surface (the rectangle at z = 0.7, Ez on output
# steps 1, 5, .., 29) and a field output volume (the Debye block, Ey)
FIELDS = test_inp.ALL_OUTPUTS + """Output_surface_list
1
1
3
1
Ez
output_timestep_information
1
30
4
Output_volume_list
1
1
1
Ey
"""


def test_surface_and_volume_field_files(tmp_path):
    paths, p, t = oracle_files(str(tmp_path), "fields", FIELDS.splitlines())
    names = sorted(os.path.basename(x) for x in paths)
    assert "fields.surface_field.tout" in names and "fields.volume_field.tout" in names
    sf = open(os.path.join(str(tmp_path), "fields.surface_field.tout")).read().splitlines()
    n_faces = len(p.spec.output_surfaces[0].faces())
    assert sf[:2] == ["# NUMBER OF OUTPUT SURFACES", "           1"]
    assert sf[4] == f"{4 * n_faces:10d}" and sf[8] == f"{8:10d}"  # 8 frames: steps 1, 5, .., 29
    assert sf.count("# START OF SURFACE FIELD OUTPUT DATA") == 8
    want = oracle.output_surfaces(t)[0]
    start = sf.index("# START OF SURFACE FIELD OUTPUT DATA")
    got = np.array([float(x) for x in sf[start + 8:start + 8 + n_faces]])
    np.testing.assert_allclose(got, want[0], rtol=1.01e-5, atol=1e-30)
    vf = open(os.path.join(str(tmp_path), "fields.volume_field.tout")).read().splitlines()
    n_cells = int((p.spec.output_volumes[-1].mask(p.spec)).sum())
    assert vf[4] == f"{24 * n_cells:10d}" and vf[8] == f"{int(t['n_timesteps']):10d}"
    assert vf.count("# START OF VOLUME FIELD OUTPUT DATA") == int(t["n_timesteps"])


def test_field_tout_from_the_huygens_input(tmp_path):
    lines = test_inp.inputs()["huygens_box"]
    paths, p, t = oracle_files(str(tmp_path), "huygens_test", lines)
    # the input also has three output surfaces and three field output volumes
    assert [os.path.basename(x) for x in paths] == ["huygens_test.excitation.tout", "huygens_test.field.tout",
                                                    "huygens_test.surface_field.tout",
                                                    "huygens_test.volume_field.tout"]
    exc, path = paths[:2]
    e = read_tout(exc)  # the Gaussian at every step, (ts-1)*dt, not flushed below 1e-30
    assert e.shape == (120, 3) and set(e[:, 1]) == {1.0}
    np.testing.assert_allclose(e[:, 2], np.asarray(t["fn_value"]).reshape(-1), rtol=5.01e-7, atol=0)
    np.testing.assert_allclose(e[:, 0], np.arange(120) * t["dt"], rtol=5.01e-7)
    with open(path) as f:
        head = [next(f).rstrip("\n") for _ in range(3)]
    assert head == ["# Time Domain Data", "# Number of data points:         30",
                    "# Number of Timesteps  :        120"]
    d = read_tout(path)
    assert d.shape == (30 * 120, 3)
    # each step: the 6 centre points at (ts-1)*dt, then the 24 face points half a step later
    assert list(d[:6, 1]) == [1, 6, 11, 16, 21, 26] and d[6, 1] == 2 and d[6, 0] > d[0, 0]
    for k, comp in zip((1, 6, 11, 16, 21, 26), ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")):
        got = d[d[:, 1] == k, 2]
        g = np.load(os.path.join(HERE, "golden", f"huygens_box_{comp}.npz"))
        assert np.linalg.norm(got - g["value"]) / np.linalg.norm(g["value"]) < TOL, comp


def test_volume_average_and_peak_files(tmp_path):
    lines = test_inp.ALL_OUTPUTS.splitlines()
    paths, p, t = oracle_files(str(tmp_path), "all", lines)
    names = sorted(os.path.basename(x) for x in paths)
    assert names == ["all.excitation.tout", "all.far_field.fout.1", "all.field.tout",
                     "all.frequency_domain_power_surface.fout", "all.frequency_output_surface.fout",
                     "all.rcs.fout", "all.rcs.tout", "all.volume_average_field.tout", "all.volume_peak_field.tout"]
    pw = [x for x in open(os.path.join(str(tmp_path), "all.frequency_domain_power_surface.fout")).read().splitlines()]
    assert pw[:3] == ["# Frequency Domain Data", "# Number of data points:         1",
                      "# Number of frequencies:         3"] and len(pw) == 6
    avg = read_tout(os.path.join(str(tmp_path), "all.volume_average_field.tout"))
    peak = read_tout(os.path.join(str(tmp_path), "all.volume_peak_field.tout"))
    dt = float(t["dt"])
    # the average runs on steps 2, 5, ..., 20 (output_timestep_information 2 20 3), the peak every step
    assert np.allclose(avg[:, 0] / dt + 1, np.arange(2, 21, 3)) and set(avg[:, 1]) == {1.0}
    assert len(peak) == int(t["n_timesteps"]) and set(peak[:, 1]) == {1.0}
    want = oracle.output_volumes(t, oracle.Oracle(t).run(t["n_timesteps"]))
    np.testing.assert_allclose(avg[:, 2], want[0], rtol=TOL, atol=1e-30)
    np.testing.assert_allclose(peak[:, 2], want[1], rtol=TOL, atol=1e-30)


def test_runner_refuses_sar_in_a_dispersive_material_before_running(tmp_path):
    """SAR only in a material of constant permittivity without magnetic
    conductivity: the reference stops at initialisation
    (SAR_volumes.F90:150-190), and so does the runner, before it needs a GPU."""
    problem_dir(str(tmp_path), "sar", test_inp.ALL_OUTPUTS.splitlines())
    with pytest.raises(ValueError, match="SAR in a dispersive dielectric material"):
        runner.run("sar", directory=str(tmp_path))


def test_runner_stops_cleanly_without_a_gpu(tmp_path):
    import torch

    from ggi_tlm_b200 import build

    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU test runs the problem")
    build.build()
    d = problem_dir(str(tmp_path), "huygens_test", test_inp.inputs()["huygens_box"])
    env = dict(os.environ, PYTHONPATH=REPO + os.pathsep + os.environ.get("PYTHONPATH", ""))
    res = subprocess.run([sys.executable, "-m", "ggi_tlm_b200.run", "huygens_test"], cwd=d, env=env,
                         capture_output=True, text=True, timeout=600)
    assert res.returncode == 1
    assert "ERROR in run_TLM_gpu:" in res.stderr
    assert not os.path.exists(os.path.join(d, "huygens_test.field.tout"))


@pytest.mark.gpu
@pytest.mark.parametrize("name, text", [("huygens_test", None), ("all", "all"), ("fields", "fields")])
def test_gpu_runner_files_match_oracle_files(gpu_lib, tmp_path, name, text):
    # without the SAR volume, which sits in a Debye material (refused, as the reference stops on it)
    lines = (test_inp.inputs()["huygens_box"] if text is None else
             (FIELDS if text == "fields" else test_inp.ALL_OUTPUTS).split("SAR_volume_list")[0].splitlines())
    run_dir, ref_dir = str(tmp_path / "run"), str(tmp_path / "oracle")
    os.makedirs(run_dir)
    os.makedirs(ref_dir)
    problem_dir(run_dir, name, lines)
    got = runner.run(name, chunk=37, directory=run_dir)
    want, _, _ = oracle_files(ref_dir, name, lines)
    assert sorted(os.path.basename(x) for x in got) == sorted(os.path.basename(x) for x in want)
    for a in want:
        b = os.path.join(run_dir, os.path.basename(a))
        with open(a) as fa, open(b) as fb:
            la, lb = fa.read().splitlines(), fb.read().splitlines()
        assert la[:3] == lb[:3] and len(la) == len(lb)
        if a.endswith("_field.tout") and (".surface_" in a or ".volume_field" in a):
            # templates and framing line for line; values to the file's 5 digits
            num = [k for k, x in enumerate(la) if not x.startswith("#") and len(x.split()) == 1 and "." in x]
            skip = set(num)
            assert [x for k, x in enumerate(la) if k not in skip] == [x for k, x in enumerate(lb) if k not in skip]
            va, vb = np.array([float(la[k]) for k in num]), np.array([float(lb[k]) for k in num])
            np.testing.assert_allclose(vb, va, rtol=1.01e-5, atol=1e-9 * max(np.abs(va).max(), 1e-300))
            continue
        if a.endswith(".frequency_output_surface.fout"):
            # template line for line; each face's cell, then its phasor to the file's 8 digits
            num = [k for k, x in enumerate(la) if len(x.split()) == 6]
            skip = set(num)
            assert [x for k, x in enumerate(la) if k not in skip] == [x for k, x in enumerate(lb) if k not in skip]
            da, db = np.loadtxt([la[k] for k in num], ndmin=2), np.loadtxt([lb[k] for k in num], ndmin=2)
            assert np.array_equal(da[:, :3], db[:, :3])
            np.testing.assert_allclose(db[:, 3:5], da[:, 3:5], rtol=1.01e-7, atol=1e-9 * np.abs(da[:, 3:5]).max())
            continue
        if ".far_field.fout" in a or ".rcs." in a:
            # comment lines as they are; the numbers to the files' printed digits
            ka = [k for k, x in enumerate(la) if x.lstrip().startswith("#")]
            assert [la[k] for k in ka] == [lb[k] for k in ka]
            da = np.loadtxt([x for x in la if not x.lstrip().startswith("#")], ndmin=2)
            db = np.loadtxt([x for x in lb if not x.lstrip().startswith("#")], ndmin=2)
            np.testing.assert_allclose(db, da, rtol=1.01e-5, atol=1e-9 * np.abs(da).max())
            continue
        if a.endswith(".fout"):
            da, db = np.loadtxt(la, comments="#", ndmin=2), np.loadtxt(lb, comments="#", ndmin=2)
            np.testing.assert_allclose(db[:, 2:4], da[:, 2:4], rtol=1.01e-6, atol=1e-9 * np.abs(da[:, 2:4]).max())
            continue
        da, db = read_tout(a), read_tout(b)
        assert np.array_equal(da[:, 1], db[:, 1])
        np.testing.assert_allclose(db[:, 0], da[:, 0], rtol=1e-7)
        # printed to 7 digits: one unit in the last digit is up to 1e-6 relative; round-off-level values
        # (components zero by symmetry) are held to an absolute floor below the file's largest value
        np.testing.assert_allclose(db[:, 2], da[:, 2], rtol=1.01e-6, atol=1e-9 * np.abs(da[:, 2]).max())
