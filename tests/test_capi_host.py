"""C-ABI library checks that need no GPU: it loads, exports every declared
symbol, fails loudly without a device, and its host-side field IO matches the
reference's IO::FieldIO."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            txt = open(os.path.join(inc, fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(glac_\w+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    import glac_b200
    lib = ctypes.CDLL(glac_b200.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_create_rejects_bad_descriptors():
    import glac_b200 as g
    for dims in [(4, 4, 4, 3), (2, 4, 4, 4), (5, 4, 4, 4)]:
        with pytest.raises(g.GlacError) as e:
            g.Lattice(dims)
        assert e.value.status in (g.GLAC_ERR_ARG, g.GLAC_ERR_CUDA)
        if e.value.status == g.GLAC_ERR_ARG:
            assert "even" in str(e.value)
    # size limits are checked before any device call: V <= 2^29, 32-bit field
    # offsets (FP64 V < 1.19e8, FP32 V < 2.68e8), Nt <= 1024
    for dims, prec, words in [((512, 512, 512, 8), "fp32", "2^29"),
                              ((256, 256, 256, 8), "fp64", "32-bit"),
                              ((512, 256, 256, 8), "fp32", "32-bit"),
                              ((4, 4, 4, 1026), "fp64", "Nt")]:
        with pytest.raises(g.GlacError) as e:
            g.Lattice(dims, precision=prec)
        assert e.value.status == g.GLAC_ERR_ARG and words in str(e.value), str(e.value)
    from glac_b200.ensemble import Ensemble
    with pytest.raises(g.GlacError) as e:
        Ensemble([(4, 4, 4, 8), (512, 256, 256, 8)], [6.0, 6.0], precision="fp32")
    assert e.value.status == g.GLAC_ERR_ARG and "lattice 1" in str(e.value)


def test_no_cpu_fallback_without_device():
    import glac_b200 as g
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(g.GlacError) as e:
        g.Lattice((4, 4, 4, 4))
    assert e.value.status == g.GLAC_ERR_CUDA


def test_field_io_roundtrip_and_reference_compat(tmp_path, oracle, reference):
    import glac_b200 as g
    N = (4, 4, 4, 8)
    reference.configure(4, 8)
    L = oracle.haar_field(N, 31)
    p = str(tmp_path / "cfg.bin")
    g.write_field(p, N, L)
    assert os.path.getsize(p) == int(np.prod(N)) * 4 * 18 * 8
    assert np.array_equal(g.read_field(p, N), L)
    # the reference's loader reads our file, and our loader reads the reference's writer
    assert np.array_equal(reference.load_field(p), L)
    reference.write_field(L, str(tmp_path), "b")
    written = [f for f in os.listdir(tmp_path / "b" / "field_configurations")]
    assert len(written) == 1
    assert np.array_equal(g.read_field(str(tmp_path / "b" / "field_configurations" / written[0]), N), L)


def test_chroma_byte_swapped_field(tmp_path, oracle, reference):
    import glac_b200 as g
    N = (4, 4, 4, 4)
    reference.configure(4, 4)
    L = oracle.haar_field(N, 8)
    p = str(tmp_path / "native.bin")
    g.write_field(p, N, L)
    raw = np.fromfile(p, dtype="<f8").astype(">f8")
    q = str(tmp_path / "chroma.bin")
    raw.tofile(q)
    assert np.array_equal(g.read_field(q, N, chroma=True), L)
    assert np.array_equal(reference.load_field(q, chroma=True), L)


def test_field_io_errors(tmp_path):
    import glac_b200 as g
    with pytest.raises(g.GlacError) as e:
        g.read_field(str(tmp_path / "missing.bin"), (4, 4, 4, 4))
    assert e.value.status == g.GLAC_ERR_IO and "does not exist" in str(e.value)
    short = tmp_path / "short.bin"
    short.write_bytes(b"\0" * 100)
    with pytest.raises(g.GlacError) as e:
        g.read_field(str(short), (4, 4, 4, 4))
    assert e.value.status == g.GLAC_ERR_IO and "expected" in str(e.value)


def test_ensemble_draw_is_seeded_and_uneven():
    from glac_b200.ensemble import BETAS, SIZES, draw_ensemble
    d1, b1 = draw_ensemble(20261203, 64)
    d2, b2 = draw_ensemble(20261203, 64)
    assert d1 == d2 and b1 == b2 and len(d1) == 64
    assert set(d1) <= set(SIZES) and set(b1) <= set(BETAS)
    assert len(set(d1)) == 4 and len(set(b1)) == 4  # every size and coupling occurs
