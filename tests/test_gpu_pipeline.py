"""Overlapped sampling + backmap + host copy (GPU): the chunked job gives the
same reaction-space samples as one naja_chr_run followed by the backmap."""
import numpy as np
import pytest

from naja_b200 import Polytope, backmap, synth
from naja_b200.pipeline import chunk_samples, sample_backmapped

pytestmark = pytest.mark.gpu


def test_chunk_rule():
    assert chunk_samples(12500, 116, 2048) % 512 == 0  # lcm(2048, 116) = 512 samples of 116 steps
    assert chunk_samples(100, 7, 0) == 100
    assert chunk_samples(100, 7, 64, rng="mrg") == 100


@pytest.mark.parametrize("sparse", ["auto", "dense"])
def test_chunked_job_equals_one_launch(cuda, sparse):
    import torch

    g = synth.genome_shaped(n=600, d=150, density=0.08, seed_T=7, seed_u=8)
    P = Polytope(g["A"], g["b"])
    nspc, thin, nch, K = 96, 8, 6, 64  # chunks of 32 samples = 4 resync periods
    kw = dict(seed=3, pair_prob=0.3, precision="fp32", sparse=sparse)
    out = torch.empty((nspc * nch, g["T"].shape[0]), dtype=torch.float32).pin_memory()
    xf = sample_backmapped(P, g["T"], g["shift"], g["start"], nspc, thin, nch, out, mode="tf32x3", chunk=32,
                           resync_interval=K, **kw)
    Y = torch.empty((nspc * nch, g["T"].shape[1]), dtype=torch.float32, device=cuda)
    xf1 = np.zeros((nch, g["T"].shape[1]))
    P.run(g["start"], nspc, thin, nch, out=Y, X_final=xf1, resync_interval=K, **kw)
    ref = backmap(g["T"], g["shift"], Y, mode="tf32x3", out=torch.empty((nspc * nch, g["T"].shape[0]),
                                                                        dtype=torch.float32, device=cuda))
    torch.cuda.synchronize()
    assert torch.equal(out, ref.cpu())
    assert np.array_equal(xf.cpu().numpy(), xf1)


@pytest.mark.parametrize("mode", ["fp64", "bf16x3"])
def test_device_outputs_and_samples(cuda, mode):
    """V and the samples in device memory (no copies), pageable numpy T / shift,
    another backmap mode: the same rows as one launch followed by the backmap."""
    import torch

    g = synth.genome_shaped(n=300, d=90, density=0.1, seed_T=9, seed_u=10)
    P = Polytope(g["A"], g["b"])
    nspc, thin, nch, K = 60, 6, 5, 36  # chunks of 18 samples = 3 resync periods, last chunk partial
    kw = dict(seed=4, pair_prob=0.3, precision="fp32")
    n, d = g["T"].shape
    out = torch.empty((nspc * nch, n), dtype=torch.float32, device=cuda)
    S = torch.empty((nspc * nch, d), dtype=torch.float32, device=cuda)
    sample_backmapped(P, g["T"], g["shift"], g["start"], nspc, thin, nch, out, mode=mode, chunk=18,
                      resync_interval=K, samples=S, **kw)
    Y = P.run(g["start"], nspc, thin, nch, resync_interval=K, **kw)
    assert np.array_equal(S.cpu().numpy(), Y)
    ref = backmap(g["T"], g["shift"], Y, mode=mode)
    assert np.array_equal(out.cpu().numpy(), ref)


def test_pageable_host_output_and_rejections(cuda):
    g = synth.genome_shaped(n=200, d=60, density=0.1, seed_T=11, seed_u=12)
    P = Polytope(g["A"], g["b"])
    nspc, thin, nch = 40, 5, 3
    out = np.empty((nspc * nch, g["T"].shape[0]), dtype=np.float64)
    sample_backmapped(P, g["T"], g["shift"], g["start"], nspc, thin, nch, out, mode="fp64", chunk=10,
                      resync_interval=25, seed=1)
    Y = P.run(g["start"], nspc, thin, nch, resync_interval=25, seed=1)
    assert np.array_equal(out, backmap(g["T"], g["shift"], Y, mode="fp64", out_dtype=np.float64))
    from naja_b200._lib import InvalidArgument

    with pytest.raises(InvalidArgument):  # a chunk of 7 samples is not a whole number of resync periods
        sample_backmapped(P, g["T"], g["shift"], g["start"], nspc, thin, nch, out, mode="fp64", chunk=7,
                          resync_interval=25, seed=1)
    with pytest.raises(InvalidArgument):  # MRG streams cannot be chunked
        sample_backmapped(P, g["T"], g["shift"], g["start"], nspc, thin, nch, out, mode="fp64", chunk=10,
                          resync_interval=25, rng="mrg")
