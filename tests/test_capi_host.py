"""The C ABI library and the host logic, without running compute (CPU)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from naja_b200 import _lib, synth

ROOT = Path(__file__).resolve().parent.parent


def _declared_functions(header="naja_chr.h"):
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(naja_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _declared_functions()
    assert "naja_chr_run" in declared and "naja_backmap" in declared
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_lib.EXPORTED)
    mlp = _declared_functions("naja_mlp.h")
    assert "naja_gemm_bf16" in mlp
    for name in mlp:
        assert hasattr(lib, name), name
    assert set(mlp) == set(_lib.EXPORTED_MLP)


def test_gemm_epilogue_struct_layout():
    E = _lib.GemmEpilogue
    assert E.c_f32.offset == 8 and E.act.offset == 24 and E.act_t.offset == 40 and E.gelu.offset == 52
    assert C.sizeof(E) == 56


def test_params_default_matches_reference_defaults():
    lib = _lib.load()
    p = _lib.ChrParams()
    lib.naja_chr_params_default(C.byref(p))
    # gpusamplers.h:30-46: seed 0, pair_prob 0, resync 0, ksparse_prob 0, ksparse_k 8, pair_mode 1
    assert (p.seed, p.pair_prob, p.resync_interval, p.ksparse_prob, p.ksparse_k, p.pair_mode) == (0, 0.0, 0, 0.0, 8, 1)
    assert (p.precision, p.rng, p.out_dtype, p.tpb) == (_lib.PREC_FP32, _lib.RNG_PHILOX, _lib.DTYPE_F32, 0)


def test_params_struct_layout():
    # offsets of the C struct on x86-64 (ints 4, doubles/pointers 8, natural alignment)
    P = _lib.ChrParams
    assert P.seed.offset == 16 and P.pair_prob.offset == 24 and P.ksparse_prob.offset == 40
    assert P.pair_i.offset == 56 and P.n_pairs.offset == 88 and P.step_offset.offset == 112
    assert P.cluster.offset == 144 and P.sparse.offset == 148 and P.slack_final.offset == 152
    assert C.sizeof(P) == 160


def test_version_string():
    assert b"sm_100a" in _lib.load().naja_version()


def test_no_device_reports_error_instead_of_crashing():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from naja_b200 import Polytope

    A, b, x0 = synth.cube(3)
    with pytest.raises(_lib.NajaError):
        Polytope(A, b)


def test_genome_generator_shape_and_start():
    g = synth.genome_shaped(n=2600, d=700)
    assert g["A"].shape == (5200, 700) and g["b"].shape == (5200,)
    nnz = (g["T"] != 0).mean()
    assert 0.075 < nnz < 0.085
    assert (g["u"] >= 1).all() and (g["u"] <= 1000).all()
    assert np.all(g["A"] @ g["start"] <= g["b"])
    assert np.all((g["T"] != 0).any(axis=0))


def test_conditioned_variants_follow_extra_row_rule():
    g = synth.genome_shaped(n=300, d=60)
    vs = synth.conditioned_variants(g, 8, max_reactions=20)
    for v in vs:
        k = len(v["tightened"])
        assert v["extra_A"].shape == (2 * k, 60)
        # y = 0 stays strictly feasible: rhs of every extra row is positive
        assert np.all(v["extra_b"] > 0)
        assert np.all(v["u_new"] <= g["u"]) and np.all(v["l_new"] >= g["l"])
