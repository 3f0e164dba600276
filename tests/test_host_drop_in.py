"""The GLAC-compatible driver (glac_b200/bin/GLAC): same JSON run-config as the
reference's createJobs.py writes, same output files (observables/, flow_observables/,
field_configurations/), physics through the C ABI on the GPU."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, assert_obs_close

GLAC = os.path.join(ROOT, "glac_b200", "bin", "GLAC")


def make_config(tmp, **over):
    """The key set of createJobs.py _create_json (createJobs.py:257-341)."""
    cfg = {"NSpatial": 4, "NTemporal": 8, "subDims": [], "beta": 6.0, "NCf": 3, "NCor": 5, "NTherm": 10,
           "NFlows": 4, "NUpdates": 10, "outputFolder": "/output/", "inputFolder": "/input/",
           "storeConfigurations": True, "storeThermalizationObservables": False, "load_config_and_run": "",
           "config_start_number": 0, "verbose": False, "pwd": str(tmp), "batchName": "t1", "hotStart": True,
           "RSTHotStart": False, "expFunc": "morningstar", "action": "wilson", "observables": ["plaq"],
           "flowObservables": ["plaq", "topc", "energy", "topct"], "load_field_configs": False,
           "chroma_config": False, "field_configs": [], "unitTesting": False, "unitTestingVerbose": False,
           "uTestFieldGaugeInvarince": "", "performanceTesting": False, "NExpTests": 1000000,
           "NRandTests": 1000000, "NDerivativeTests": 100, "TaylorPolDegree": 8, "SU3Eps": 0.24,
           "flowEpsilon": 0.01, "metropolisSeed": 12, "randomMatrixSeed": 13, "samplingFrequency": 25,
           "debug": False}
    cfg.update(over)
    path = os.path.join(str(tmp), "config_%s.json" % cfg["batchName"])
    with open(path, "w") as f:
        json.dump(cfg, f, indent=4)
    return path, cfg


def test_print_config_parses_job_driver_json(tmp_path):
    path, cfg = make_config(tmp_path, precision="fp32", reunitInterval=5)
    out = subprocess.run([GLAC, "--print-config", path], capture_output=True, text=True, check=True).stdout
    p = json.loads(out)
    for k in ("NSpatial", "NTemporal", "NCf", "NCor", "NTherm", "NFlows", "NUpdates", "beta", "flowEpsilon",
              "metropolisSeed", "randomMatrixSeed", "expFunc", "observables", "flowObservables", "batchName"):
        assert p[k] == cfg[k], k
    assert p["precision"] == "fp32" and p["reunitInterval"] == 5


def test_config_errors(tmp_path):
    path, _ = make_config(tmp_path)
    cfg = json.load(open(path))
    del cfg["beta"]
    json.dump(cfg, open(path, "w"))
    r = subprocess.run([GLAC, "--print-config", path], capture_output=True, text=True)
    assert r.returncode != 0 and "'beta' is missing" in r.stdout
    r = subprocess.run([GLAC, "--print-config", str(tmp_path / "nope.json")], capture_output=True, text=True)
    assert r.returncode != 0 and "does not exist" in r.stdout
    path, _ = make_config(tmp_path, action="improved")
    r = subprocess.run([GLAC, "--print-config", path], capture_output=True, text=True)
    assert r.returncode != 0 and "not recognized" in r.stdout


def read_flow(path):
    lines = open(path).read().split("\n")
    assert lines[0].startswith("beta ") and lines[1].startswith("NFlows ") and lines[2].startswith("FlowEpsilon ")
    return np.array([[float(x) for x in ln.split()] for ln in lines[3:] if ln.strip()])


@pytest.mark.gpu
def test_generate_flow_and_write_like_the_reference(tmp_path, oracle):
    path, cfg = make_config(tmp_path)
    r = subprocess.run([GLAC, path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = tmp_path / "output" / "t1"
    N = (4, 4, 4, 8)
    for i in range(3):
        fn = out / "field_configurations" / ("t1_b6.000000_N4_NT8_np1_config%05d.bin" % i)
        assert fn.exists()
        import glac_b200 as g
        links = g.read_field(str(fn), N)
        obs0 = oracle.observables(N, links)
        flowed = oracle.flow(N, links, 0.01, 4)
        obs4 = oracle.observables(N, flowed)
        plaq = read_flow(out / "flow_observables" / "plaq" / ("t1_plaq_flow_config%05d.dat" % i))
        topc = read_flow(out / "flow_observables" / "topc" / ("t1_topc_flow_config%05d.dat" % i))
        energy = read_flow(out / "flow_observables" / "energy" / ("t1_energy_flow_config%05d.dat" % i))
        topct = read_flow(out / "flow_observables" / "topct" / ("t1_topct_flow_config%05d.dat" % i))
        assert plaq.shape == (5, 2) and topct.shape == (5, 1 + 8)
        assert np.allclose(plaq[:, 0], 0.01 * np.arange(5))
        # files print 15 decimals: 1e-11 relative leaves room for the last digit of q(t) ~ 1e-3
        assert_obs_close([plaq[0, 1], topc[0, 1], energy[0, 1]], obs0[:3], 1e-12, "t = 0", slices=())
        assert_obs_close(np.r_[plaq[4, 1], topc[4, 1], energy[4, 1], topct[4, 1:]], obs4, 1e-11, "t = 0.04")
    txt = open(out / "observables" / "plaq_t1.dat").read().split("\n")
    assert txt[0] == "beta 6" and txt[1].startswith("acceptanceCounter ")
    assert txt[2] == "NCor 5" and txt[3] == "NCf 3" and txt[4] == "NTherm 10"
    vals = [float(x) for x in txt[8:] if x.strip()]
    assert len(vals) == 3
    assert abs(float(txt[5].split()[1]) - np.mean(vals)) < 1e-14


@pytest.mark.gpu
def test_load_and_flow_matches_reference(tmp_path, oracle, reference):
    N = (4, 4, 4, 8)
    links = oracle.haar_field(N, 77)
    import glac_b200 as g
    os.makedirs(tmp_path / "input")
    g.write_field(str(tmp_path / "input" / "cfgA.bin"), N, links)
    path, cfg = make_config(tmp_path, load_field_configs=True, field_configs=["cfgA.bin"], NFlows=3,
                            batchName="t2", flowObservables=["plaq", "topc", "energy"])
    r = subprocess.run([GLAC, path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    reference.configure(4, 8, flow_eps=0.01, nflows=3)
    flowed = reference.flow(links, 3)
    want = reference.observables(flowed)
    out = tmp_path / "output" / "t2" / "flow_observables"
    got = [read_flow(out / n / ("t2_%s_flow_config00000.dat" % n))[3, 1] for n in ("plaq", "topc", "energy")]
    assert_obs_close(got, want[:3], 1e-12, "after 3 steps", slices=())
    assert not (out / "topct").exists()


@pytest.mark.gpu
def test_energy_topc_field_density_run(tmp_path, oracle, reference):
    # flowObservables ["energyTopcFieldDensity"] alone: LatticeActionChargeDensity
    # with per-site q and E fields every samplingFrequency flow steps, one config
    N, V = (4, 4, 4, 8), 512
    links = oracle.haar_field(N, 78)
    import glac_b200 as g
    os.makedirs(tmp_path / "input")
    g.write_field(str(tmp_path / "input" / "cfgB.bin"), N, links)
    path, cfg = make_config(tmp_path, load_field_configs=True, field_configs=["cfgB.bin"], NFlows=4,
                            batchName="t3", flowObservables=["energyTopcFieldDensity"], samplingFrequency=2)
    r = subprocess.run([GLAC, path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    sf = tmp_path / "output" / "t3" / "scalar_fields"
    reference.configure(4, 8, flow_eps=0.01, nflows=4)
    for step in (0, 2, 4):
        name = "t3_b6.000000_N4_NT8_np1_config%05d.bin" % step
        q = np.fromfile(sf / "topc" / name, dtype=np.float64)
        e = np.fromfile(sf / "energy" / name, dtype=np.float64)
        assert q.size == V and e.size == V
        qr, er, _ = reference.density(reference.flow(links, step) if step else links)
        assert np.max(np.abs(q - qr)) < 1e-12 * np.max(np.abs(qr))
        assert np.max(np.abs(e - er)) < 1e-12 * np.max(np.abs(er))
    for step in (1, 3):
        assert not (sf / "topc" / ("t3_b6.000000_N4_NT8_np1_config%05d.bin" % step)).exists()
    fo = tmp_path / "output" / "t3" / "flow_observables"
    topc = read_flow(fo / "topc" / "t3_topc_flow_config00000.dat")
    q4 = np.fromfile(sf / "topc" / "t3_b6.000000_N4_NT8_np1_config00004.bin", dtype=np.float64)
    assert abs(topc[4, 1] - q4.sum()) < 1e-12
    assert not (fo / "topct").exists()


@pytest.mark.gpu
def test_stored_configuration_carries_its_random_stream(tmp_path):
    # a chain stopped after config 0 and resumed from its file continues with the
    # same random numbers as the uninterrupted chain
    path, cfg = make_config(tmp_path, NCf=2, NCor=3, NTherm=4, NFlows=0, batchName="t4")
    r = subprocess.run([GLAC, path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    fc = tmp_path / "output" / "t4" / "field_configurations"
    side = open(fc / "t4_b6.000000_N4_NT8_np1_config00000.bin.rng").read().split()
    assert side[0] == "metropolisSeed" and float(side[1]) == 12 and side[2] == "sweep" and int(side[3]) == 4 + 3
    os.makedirs(tmp_path / "input")
    import shutil
    for ext in ("", ".rng"):
        shutil.copy(fc / ("t4_b6.000000_N4_NT8_np1_config00000.bin" + ext), tmp_path / "input" / ("c0.bin" + ext))
    path2, _ = make_config(tmp_path, NCf=1, NCor=3, NTherm=0, NFlows=0, batchName="t5", load_config_and_run="c0.bin")
    r = subprocess.run([GLAC, path2], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    import glac_b200 as g
    N = (4, 4, 4, 8)
    a = g.read_field(str(fc / "t4_b6.000000_N4_NT8_np1_config00001.bin"), N)
    b = g.read_field(str(tmp_path / "output" / "t5" / "field_configurations" / "t5_b6.000000_N4_NT8_np1_config00000.bin"), N)
    assert np.array_equal(a, b)


@pytest.mark.gpu
def test_weinberg_sampler_files_match_reference(tmp_path, oracle, reference):
    N = (4, 4, 4, 8)
    links = oracle.haar_field(N, 79)
    import glac_b200 as g
    os.makedirs(tmp_path / "input")
    g.write_field(str(tmp_path / "input" / "cfgW.bin"), N, links)
    path, cfg = make_config(tmp_path, load_field_configs=True, field_configs=["cfgW.bin"], NFlows=3,
                            batchName="t6", flowObservables=["plaq", "topc", "energy", "weinberg"])
    r = subprocess.run([GLAC, path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    reference.configure(4, 8, flow_eps=0.01, nflows=3)
    want = reference.supersampler(reference.flow(links, 3))
    fo = tmp_path / "output" / "t6" / "flow_observables"
    row = {n: read_flow(fo / n / ("t6_%s_flow_config00000.dat" % n))[3, 1:] for n in
           ("plaq", "topc", "energy", "weinberg", "topct", "weinbergt")}
    got = np.concatenate([row["plaq"], row["topc"], row["energy"], row["weinberg"], row["topct"], row["weinbergt"]])
    assert_obs_close(got, want, 1e-11, "weinberg files", scalars=("plaq", "topc", "energy", "weinberg"),
                     slices=("topct", "weinbergt"))
