"""Device pointers of another GPU are rejected before any kernel runs (GPU).

A kernel launched on the current device would fault on plain device memory
of another device unless peer access happened to be enabled; the C ABI
returns NAJA_ERR_INVALID_ARGUMENT instead.  Needs two visible GPUs.
"""
import numpy as np
import pytest

from naja_b200 import Polytope, backmap, synth
from naja_b200._lib import InvalidArgument

pytestmark = pytest.mark.gpu


def test_pointer_of_another_device_is_rejected(cuda):
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    other = torch.device("cuda", 1)
    g = synth.genome_shaped(n=60, d=20, density=0.2, seed_T=1, seed_u=2)
    P = Polytope(g["A"], g["b"], device=0)
    X_other = torch.zeros((3, 20), dtype=torch.float64, device=other)
    with torch.cuda.device(0):
        with pytest.raises(InvalidArgument, match="another GPU"):
            P.run(X_other, 5, 2, 3, stream=None)
        Y_other = torch.zeros((4, 20), dtype=torch.float32, device=other)
        with pytest.raises(InvalidArgument, match="another GPU"):
            backmap(g["T"], g["shift"], Y_other, mode="fp64", out=np.empty((4, 60), dtype=np.float32))
    P.close()
