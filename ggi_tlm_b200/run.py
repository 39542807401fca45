"""Run a GGI_TLM problem file on the GPU and write its time-domain results.

    python -m ggi_tlm_b200.run <problem_name> [--fp32] [--device N] [--chunk STEPS]

As the reference's GGI_TLM program does (SRC/GGI_TLM.F90), this reads
``<problem_name>.inp`` from the working directory (material files resolve
against it too), runs the time loop, and writes, in the reference's format
and file names (TLM_MODULES/File_information.F90:143-158):

- ``<problem_name>.excitation.tout``: every excitation function at every
  timestep (excitation.F90:186-553);
- ``<problem_name>.field.tout``: the output points, each on its own output
  steps (output_points.F90);
- ``<problem_name>.frequency_domain_power_surface.fout``: the power through
  each power surface at each of its frequencies
  (frequency_domain_power_surfaces.F90:420-574);
- ``<problem_name>.volume_average_field.tout`` and
  ``.volume_peak_field.tout``: one value per output volume average or peak
  and output step (output_volume_averages.F90:330-350,
  output_volume_peak.F90:320-340), numbered within their own packet;
- ``<problem_name>.far_field.fout.<k>``: the far-field pattern of each
  far-field surface (far_field_surfaces.F90:370-712, ``postprocess``);
- ``<problem_name>.SAR.fout``: the SAR of each SAR volume
  (SAR_volumes.F90:334-622, ``postprocess``);
- ``<problem_name>.rcs.tout`` and ``.rcs.fout``: the RCS surface's far
  field in time and its RCS spectrum (RCS_surfaces.F90:575-762,
  ``postprocess``);
- ``<problem_name>.surface_field.tout`` and ``.volume_field.tout``: the
  frames of the output surfaces and field output volumes with their
  geometry templates (output_surfaces.F90:326-927,
  output_volumes.F90:227-745, ``postprocess``).

The run goes through the library's C ABI in chunks of ``--chunk`` steps,
reading the output points back after each chunk.  The other outputs
(surfaces, volumes, DFTs, far field, SAR, power) are returned by the
GpuMesh accessors.  Without the CUDA library or a GPU it stops with the
library's message and exit code 1.
"""
from __future__ import annotations

import argparse
import os
import sys
from typing import List, Optional, Sequence

import numpy as np

from . import capi, fout, postprocess
from .inp import InpProblem, read_inp_file
from .problem import build_tables, probe_series
from .tout import data_line, excitation_rows, field_rows, header, output_flag


def _volume_rows(t: dict, spec, values: List[np.ndarray], kind: str):
    """(time, number, value) rows of the output volumes of one kind, at the
    cell-output time (timestep-1)*dt of each step get_output_flag accepts."""
    dt = float(t["dt"])
    n = int(t["n_timesteps"])
    vols = [(k, v) for k, v in enumerate(spec.output_volumes) if v.kind == kind]
    row_of = []  # per volume: output step -> row of its result array
    for _, v in vols:
        last = n if v.last_step is None else v.last_step
        st = [ts for ts in range(1, n + 1) if output_flag(ts, (v.first_step, last, v.interval))]
        row_of.append({ts: i for i, ts in enumerate(st)})
    rows = []
    for ts in range(1, n + 1):
        for num, ((k, _), rmap) in enumerate(zip(vols, row_of), start=1):
            if ts in rmap:
                rows.append(((ts - 1) * dt, num, float(values[k][rmap[ts]])))
    return rows, len(vols)


def write_results(name: str, p: InpProblem, t: dict, cell_out: np.ndarray, face_out: np.ndarray,
                  volumes: Optional[List[np.ndarray]] = None, directory: str = ".",
                  power: Optional[np.ndarray] = None, far_field: Optional[np.ndarray] = None,
                  sar: Optional[np.ndarray] = None, rcs: Optional[np.ndarray] = None,
                  surfaces: Optional[List[np.ndarray]] = None, dft: Optional[np.ndarray] = None,
                  modes: Optional[np.ndarray] = None) -> List[str]:
    """Write the result files of a finished run; returns the paths written.
    ``cell_out`` is [steps, n_kept, 6], ``face_out`` [n_face_points, steps],
    ``volumes`` the output volume results, ``power`` the power surface
    accumulators [faces, 4], ``far_field`` the far-field accumulators
    [faces, 6], ``sar`` the SAR accumulators [cells, 3], ``rcs`` the RCS
    far field [4, points], ``surfaces`` the output surface frames, ``dft``
    the frequency output surfaces' phasors [faces, 2] and ``modes`` the mode
    outputs [modes, steps]."""
    written = []
    n = int(t["n_timesteps"])
    if int(t["n_functions"]):
        path = os.path.join(directory, name + ".excitation.tout")
        _write(path, header(int(t["n_functions"]), n), excitation_rows(t), flush_small=False)
        written.append(path)
    if p.spec.outputs:
        centre = probe_series(t, cell_out) if int(t["n_out_cells"]) else np.zeros((0, n))
        rows = field_rows(t, centre, face_out, timing=p.output_timing)
        path = os.path.join(directory, name + ".field.tout")
        _write(path, header(len(p.spec.outputs), n), rows)
        written.append(path)
    if p.spec.power_surfaces and power is not None:
        surf = [k + 1 for k, ps in enumerate(p.spec.power_surfaces) for _ in ps.frequencies]
        path = os.path.join(directory, name + ".frequency_domain_power_surface.fout")
        with open(path, "w") as f:
            for line in fout.power_surface_lines(t["ps_freq"], surf, fout.power_surfaces(t, power)):
                f.write(line + "\n")
        written.append(path)
    if p.spec.far_field_surfaces and far_field is not None:
        written += postprocess.write_far_field_surfaces(name, p.spec, t, far_field, p.post["far_field"], directory)
    if p.spec.sar_volumes and sar is not None:
        written += postprocess.write_sar_volumes(name, p.spec, t, sar, p.post["sar_density"], directory)
    if p.spec.rcs_surface is not None and rcs is not None:
        written += postprocess.write_rcs(name, t, rcs, p.post["rcs"], int(t["hs_fn"]), directory)
    written += postprocess.write_field_files(name, p.spec, t, surfaces, volumes, directory)
    if p.spec.dft_surfaces and dft is not None:
        written += postprocess.write_frequency_output_surfaces(name, p.spec, t, dft, directory)
    if p.spec.mode_outputs and modes is not None:
        # Mode_output (output_modes.F90:546-620): every step after connect, at time (timestep-1)*dt + dt/2
        dt = float(t["dt"])
        rows = [((ts - 1) * dt + dt / 2.0, k + 1, float(modes[k, ts - 1]))
                for ts in range(1, n + 1) for k in range(len(p.spec.mode_outputs))]
        path = os.path.join(directory, name + ".mode.tout")
        _write(path, header(len(p.spec.mode_outputs), n), rows)
        written.append(path)
    for kind, extn in (("average", ".volume_average_field.tout"), ("peak", ".volume_peak_field.tout")):
        if any(v.kind == kind for v in p.spec.output_volumes):
            rows, count = _volume_rows(t, p.spec, volumes, kind)
            path = os.path.join(directory, name + extn)
            _write(path, header(count, n), rows)
            written.append(path)
    return written


def _write(path: str, head: Sequence[str], rows, flush_small: bool = True) -> None:
    with open(path, "w") as f:
        for line in head:
            f.write(line + "\n")
        for time, num, value in rows:
            f.write(data_line(time, num, value, flush_small) + "\n")


def run(name: str, precision: int = capi.TLM_PRECISION_FP64, device: int = 0, chunk: int = 1000,
        directory: str = ".", lenient: bool = False) -> List[str]:
    """Read ``<directory>/<name>.inp``, run it and write its result files;
    ``lenient`` leaves out the output packets the GPU path refuses."""
    p = read_inp_file(os.path.join(directory, name + ".inp"), lenient=lenient)
    for item in p.skipped:
        if ":" in item:
            print("left out", item)
    t = build_tables(p.spec)
    n = int(t["n_timesteps"])
    postprocess.check_sar_volumes(p.spec)  # the reference stops here, before time stepping
    with capi.GpuMesh(t, precision=precision, device=device) as g:
        cells, faces = [], []
        for first in range(1, n + 1, chunk):
            k = min(chunk, n - first + 1)
            g.run(k)
            cells.append(g.cell_output(first, k))
            faces.append(g.face_output(first, k))
        cell_out = np.concatenate(cells) if cells else np.zeros((0, 0, 6))
        face_out = np.concatenate(faces, axis=1) if faces else np.zeros((0, 0))
        volumes = g.output_volumes() if p.spec.output_volumes else None
        power = g.power_surfaces() if p.spec.power_surfaces else None
        far_field = g.far_field() if p.spec.far_field_surfaces else None
        sar = g.sar_volumes() if p.spec.sar_volumes else None
        rcs = g.rcs() if p.spec.rcs_surface is not None else None
        surfaces = g.output_surfaces() if p.spec.output_surfaces else None
        dft = g.dft() if p.spec.dft_surfaces else None
        modes = g.mode_outputs(1, n) if p.spec.mode_outputs else None
    return write_results(name, p, t, cell_out, face_out, volumes, directory, power, far_field, sar, rcs, surfaces,
                         dft, modes)


def main(argv: Optional[Sequence[str]] = None) -> int:
    ap = argparse.ArgumentParser(prog="python -m ggi_tlm_b200.run", description=__doc__.split("\n")[0])
    ap.add_argument("problem_name")
    ap.add_argument("--fp32", action="store_true", help="FP32 link state (default FP64)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--chunk", type=int, default=1000, help="steps per run call between read-backs")
    ap.add_argument("--lenient", action="store_true", help="leave out output packets the GPU path refuses")
    a = ap.parse_args(argv)
    try:
        for path in run(a.problem_name, capi.TLM_PRECISION_FP32 if a.fp32 else capi.TLM_PRECISION_FP64, a.device,
                        a.chunk, lenient=a.lenient):
            print("wrote", path)
    except (RuntimeError, OSError) as e:  # TLMError is a RuntimeError, as is a library not built
        print(f"ERROR in run_TLM_gpu: {e}", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
