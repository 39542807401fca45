"""WAVEGUIDE_RESONATOR: a PEC-walled WR90-like cavity (2 x 46 x 46 cells)
driven by a soft Ex excitation surface across its cross section
(Excitation_surface_list, side -1), read from the reference's own input and
carried through its own post-processing input:

* option 3 on output point 1 (8 GHz to 12 GHz, 800 frequencies) gives
  waveguide.field.fout_ref byte for byte from the oracle's run;
* option 13 on the run's .frequency_output_surface.fout (the Ex phasor at
  9.217 GHz on a zplane) gives the mode file WR90.mode_ref byte for byte.

The reader's excitation surfaces and volumes become face and centre
sources: one side of each face (excitation_surfaces.F90:236-262), both
sides for side 0, and a centre source per cell of an excitation volume
(excitation_volumes.F90:94-126).  GPU: the library against the oracle,
including one-sided hard sources on side 2, whose type connect does not
read (it reads side 1's types on both sides)."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import inp, post_process
from ggi_tlm_b200 import run as runner
from ggi_tlm_b200.problem import SOURCE_HARD, SOURCE_SOFT, build_tables, probe_series

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import test_inp as T  # noqa: E402
import oracle  # noqa: E402


def lines(side=None, kind=None):
    """The case's input, with the excitation surface's side or source type changed."""
    src = list(T.inputs()["waveguide"])
    k = next(i for i, x in enumerate(src) if x.lower().startswith("excitation_surface_list"))
    if side is not None:
        assert "side of surface" in src[k + 5]
        src[k + 5] = f"{side}   ! side of surface for excitation"
    if kind is not None:
        assert src[k + 7].strip() == "soft"
        src[k + 7] = kind
    return src


def problem(**kw):
    p = inp.read_inp(lines(**kw), T.materials)
    return p, build_tables(p.spec)


def golden(name):
    return [str(x) for x in np.load(os.path.join(HERE, "golden", "fout_text.npz"))[name]]


def test_reader_turns_the_excitation_surface_into_one_sided_face_sources():
    p, t = problem()
    ex = p.spec.point_excitations
    assert len(ex) == 2 * 46 and all(e.one_side and e.face == "zmin" and e.cell[2] == 6 for e in ex)
    assert int(t["n_face_points"]) == 92 and set(np.asarray(t["fpt_side"]).tolist()) == {1}
    # side +1: the other side of the same faces, the max faces of the cells below
    p1, t1 = problem(side=1)
    assert all(e.face == "zmax" and e.cell[2] == 5 for e in p1.spec.point_excitations)
    assert set(np.asarray(t1["fpt_side"]).tolist()) == {2}
    assert np.array_equal(t1["fpt_face"], t["fpt_face"])
    # side 0: the faces as for -1, both sides
    p0, t0 = problem(side=0)
    assert [e.cell for e in p0.spec.point_excitations] == [e.cell for e in ex]
    assert set(np.asarray(t0["fpt_side"]).tolist()) == {0}
    with pytest.raises(ValueError, match="side must be"):
        problem(side=2)
    with pytest.raises(ValueError, match="source type"):
        problem(kind="medium")


def test_excitation_volume_is_a_centre_source_per_cell():
    """An Excitation_volume_list over a block of cells gives the tables of
    the same centre point excitations listed one by one."""
    src = list(T.inputs()["waveguide"])
    k = next(i for i, x in enumerate(src) if x.lower().startswith("excitation_surface_list"))
    vol = ["Volume_list", "1", "1", "rectangular_block2", "-0.0005 -0.0015 -0.0015  0.0005 0.0015 0.0005",
           "0.0 0.0 0.0", "0.0 0.0 0.0", "",
           "Excitation_volume_list", "1", "1", "1", "1", "Ey", "hard"]
    assert src[k + 7].strip() == "soft"
    p = inp.read_inp(src[:k] + vol + src[k + 8:], T.materials)
    ex = p.spec.point_excitations
    assert len(ex) == 2 * 6 * 4
    assert all(e.face == "centre" and e.component == "Ey" and e.source_type == SOURCE_HARD for e in ex)
    cells = sorted(e.cell for e in ex)
    assert cells == sorted((x, y, z) for x in (1, 2) for y in range(21, 27) for z in range(21, 25))
    t = build_tables(p.spec)
    assert int(t["n_exc_points"]) == len(ex) and int(t["n_face_points"]) == 0
    assert set(np.asarray(t["pt_type"]).tolist()) == {SOURCE_HARD}


def run_oracle(t):
    o = oracle.Oracle(t)
    cell = o.run(int(t["n_timesteps"]))
    return cell, o.dft()


def test_oracle_run_and_post_processing_reproduce_the_reference_files(tmp_path):
    d = str(tmp_path)
    p, t = problem()
    cell, dft = run_oracle(t)
    written = runner.write_results("waveguide", p, t, cell, np.zeros((0, int(t["n_timesteps"]))), None, d, dft=dft)
    assert os.path.basename(written[-1]) == "waveguide.frequency_output_surface.fout"
    post = [str(x) for x in np.load(os.path.join(HERE, "golden", "post_process_text.npz"))["waveguide"]]
    assert [os.path.basename(x) for x in post_process.run(post, d)] == ["waveguide.field.fout", "WR90.mode"]
    assert open(os.path.join(d, "waveguide.field.fout")).read().splitlines() == golden("waveguide")
    assert open(os.path.join(d, "WR90.mode")).read().splitlines() == golden("waveguide_mode")


def test_two_sided_and_one_sided_sources_differ_as_the_sides_do():
    """Linearity of the soft sources: side 0 excites both sides of each
    face, so its run is the sum of the side -1 and side +1 runs."""
    runs = {}
    for side in (-1, 1, 0):
        _, t = problem(side=side)
        t = dict(t, n_timesteps=600)
        runs[side] = probe_series(t, oracle.Oracle(t).run(600))
    a, b, c = (np.asarray(runs[s]) for s in (-1, 1, 0))
    assert np.linalg.norm(a - b) > 1e-3 * np.linalg.norm(a)
    assert np.linalg.norm(c - (a + b)) <= 1e-12 * np.linalg.norm(c)


@pytest.mark.gpu
@pytest.mark.parametrize("side,kind", [(-1, None), (1, "hard"), (0, "hard")])
def test_gpu_excitation_surfaces_match_the_oracle(gpu_lib, side, kind):
    from ggi_tlm_b200 import capi

    _, t = problem(side=side, kind=kind)
    n = int(t["n_timesteps"])
    cell, dft = run_oracle(t)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(n)
        got, gdft = g.cell_output(), g.dft()
    assert np.linalg.norm(got - cell) <= 1e-10 * np.linalg.norm(cell)
    assert np.linalg.norm(gdft - dft) <= 1e-10 * np.linalg.norm(dft)


@pytest.mark.gpu
def test_gpu_waveguide_through_the_runner_and_the_post_processor(gpu_lib, tmp_path):
    """``python -m ggi_tlm_b200.run waveguide`` then ``python -m
    ggi_tlm_b200.post_process`` on the case's own post-processing input: the
    spectrum and the mode file against the reference's (the GPU's FP64 series
    differ from the oracle's by ~1e-13, which can move a rare 7th printed
    digit: 99 % of the lines exact, the rest to 1e-5)."""
    import subprocess

    d = str(tmp_path)
    with open(os.path.join(d, "waveguide.inp"), "w", encoding="latin-1") as f:
        f.write("\n".join(lines()) + "\n")
    post = [str(x) for x in np.load(os.path.join(HERE, "golden", "post_process_text.npz"))["waveguide"]]
    with open(os.path.join(d, "GGI_TLM_post_process_in.txt"), "w") as f:
        f.write("\n".join(post) + "\n")
    env = dict(os.environ, PYTHONPATH=os.path.dirname(HERE))
    for cmd in (["-m", "ggi_tlm_b200.run", "waveguide"],
                ["-m", "ggi_tlm_b200.post_process", "GGI_TLM_post_process_in.txt"]):
        res = subprocess.run([sys.executable, *cmd], cwd=d, env=env, capture_output=True, text=True, timeout=600)
        assert res.returncode == 0, res.stderr[-2000:]
    for name, key, cols in (("waveguide.field.fout", "waveguide", [2, 3]), ("WR90.mode", "waveguide_mode", [3, 4])):
        got = open(os.path.join(d, name)).read().splitlines()
        gold = golden(key)
        assert len(got) == len(gold)
        assert sum(a == b for a, b in zip(got, gold)) >= 0.99 * len(gold)
        a = np.loadtxt([x for x in got if not x.startswith("#")])
        b = np.loadtxt([x for x in gold if not x.startswith("#")])
        np.testing.assert_allclose(a[:, cols], b[:, cols], rtol=1e-5, atol=1e-5 * np.abs(b[:, cols]).max())
