"""The in-reference binding of the C ABI: the reference's own program built
twice from its sources by oracle/Makefile -- unmodified (oracle/_ref/bin/GLAC)
and with GLAC/flow/flow.cpp replaced by oracle/binding/flow_glac.cpp, whose
Flow::flowField runs each RK3 step through glac_set_links / glac_flow /
glac_get_links on the GPU (oracle/_ref/bin/GLAC_bound).  Everything else is the
reference's: the JSON configuration, System's load_field_configs run mode
(GLAC/system.cpp:570-602), the MasterSamplerTopcXYZ measurement after every
step and the flow_observables files.  The same job on the same stored
configurations must give the same files: every observable of every flow step
within the FP64 bar (1e-12 per flow step taken, relative, quantity by
quantity)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, assert_obs_close
from test_host_drop_in import make_config, read_flow

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "oracle", "_ref", "bin")


def run(binary, tmp, cfg_path):
    r = subprocess.run([os.path.join(BIN, binary), cfg_path], capture_output=True, text=True, timeout=900,
                       cwd=str(tmp))
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r.stdout


def flow_table(out, batch, cfg_number, names=("plaq", "topc", "energy"), nt=None):
    """Rows per flow step: [plaq, topc, energy, topct[Nt]]."""
    cols = [read_flow(out / n / f"{batch}_{n}_flow_config{cfg_number:05d}.dat")[:, 1] for n in names]
    rows = np.stack(cols, axis=1)
    if nt:
        topct = read_flow(out / "topct" / f"{batch}_topct_flow_config{cfg_number:05d}.dat")[:, 1:]
        assert topct.shape[1] == nt
        rows = np.concatenate([rows, topct], axis=1)
    return rows


def test_bound_flow_reproduces_the_reference_job(tmp_path, oracle):
    for b in ("GLAC", "GLAC_bound"):
        if not os.path.exists(os.path.join(BIN, b)):
            pytest.skip(f"{b} not built (oracle/Makefile ref-bin ref-bin-bound needs the reference sources)")
    import glac_b200 as g
    N = (8, 8, 8, 16)
    names = []
    os.makedirs(tmp_path / "input")
    for k, seed in enumerate((11, 12)):
        with g.Lattice(N, beta=6.0, precision="fp64", seed=seed) as L:  # thermalised start fields
            L.set_links(oracle.haar_field(N, seed))
            L.metropolis(30)
            g.write_field(str(tmp_path / "input" / f"cfg{k}.bin"), N, L.get_links())
        names.append(f"cfg{k}.bin")
    tables = {}
    for b in ("GLAC", "GLAC_bound"):
        d = tmp_path / b
        os.makedirs(d / "input")
        for n in names:
            os.link(tmp_path / "input" / n, d / "input" / n)
        # the folders createJobs.py prepares before a run (createJobs.py:160-200)
        for sub in ("observables", "field_configurations", "flow_observables/plaq", "flow_observables/topc",
                    "flow_observables/energy", "flow_observables/topct"):
            os.makedirs(d / "output" / "bind" / sub)
        path, cfg = make_config(d, NSpatial=8, NTemporal=16, load_field_configs=True, field_configs=names,
                                NFlows=10, flowEpsilon=0.01, batchName="bind",
                                flowObservables=["plaq", "topc", "energy", "topct"])
        run(b, d, path)
        out = d / "output" / "bind" / "flow_observables"
        tables[b] = [flow_table(out, "bind", k, nt=N[3]) for k in range(len(names))]
    for k in range(len(names)):
        ref, bound = tables["GLAC"][k], tables["GLAC_bound"][k]
        assert ref.shape == bound.shape == (11, 3 + N[3])
        for step in range(11):
            assert_obs_close(bound[step], ref[step], max(step, 1) * 1e-12, f"config {k}, flow step {step}")
