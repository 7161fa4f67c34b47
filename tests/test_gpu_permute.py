"""Rank-N in-place permutations (t213_permute; the reference's rank-N model is
TensorUtil, src/tensor_util.cpp:7-23,79-92) against the oracle's restatement
of TensorUtil::seq_tt, and torch.ops.t213.permute_ against torch's own
permute().contiguous().  Bit-exact."""
import importlib
import itertools
import random

import numpy as np
import pytest
import torch

from conftest import from_device, to_device

pytestmark = pytest.mark.gpu


def cases():
    rng = random.Random(11)
    out = [((512, 384, 16), (1, 0, 2)), ((8, 6, 4, 2), (3, 2, 1, 0)), ((3, 5, 7, 11, 2), (4, 2, 0, 3, 1)),
           ((64, 48, 32), (2, 0, 1)), ((64, 48, 32), (1, 2, 0)), ((1, 7, 1, 9), (3, 1, 2, 0)),
           ((1000, 999), (1, 0)), ((5,), (0,)), ((4, 0, 3), (2, 1, 0)),
           # leading axes kept in place: merged into 8-16-byte elements, or
           # into 64-byte-and-larger segments moved by one cycle pass per step
           ((2, 37, 41), (0, 2, 1)), ((32, 5, 7, 3), (0, 2, 1, 3)), ((16, 3, 9), (0, 2, 1)),
           ((64, 30, 20, 6), (0, 3, 2, 1)), ((3, 5, 7), (0, 2, 1)), ((8, 4, 50, 60), (0, 1, 3, 2))]
    for _ in range(12):
        rank = rng.randint(2, 6)
        dims = tuple(rng.randint(1, 24) for _ in range(rank))
        perm = list(range(rank))
        rng.shuffle(perm)
        out.append((dims, tuple(perm)))
    return out


@pytest.mark.parametrize("eb", (4, 8, 16, 1, 2))
@pytest.mark.parametrize("dims,perm", cases(), ids=lambda v: "x".join(map(str, v)))
def test_permute_matches_oracle(cuda, oracle, t213, dims, perm, eb):
    vol = int(np.prod(dims))
    x = oracle.random_bits(vol, eb, sum(dims))
    want = oracle.seq_tt(x.view(np.dtype((np.void, eb))), list(dims), list(perm)).view(np.uint8)
    dev = to_device(cuda, x)
    t213.permute(dev, dims, perm, elem_bytes=eb)
    cuda.cuda.synchronize()
    assert np.array_equal(from_device(dev), want), (dims, perm, eb)


def test_every_permutation_of_rank4(cuda, oracle, t213):
    dims = (6, 5, 4, 3)
    x = oracle.random_bits(int(np.prod(dims)), 4, 3)
    for perm in itertools.permutations(range(4)):
        want = oracle.seq_tt(x.view(np.uint32), list(dims), list(perm)).view(np.uint8)
        dev = to_device(cuda, x)
        t213.permute(dev, dims, perm, elem_bytes=4)
        assert np.array_equal(from_device(dev), want), perm


@pytest.mark.parametrize("dims,perm", [((4, 3), (0, 0)), ((4, 3), (0, 2)), ((4, -1), (1, 0))])
def test_permute_rejects_bad_arguments(cuda, t213, dims, perm):
    dev = cuda.zeros(64, dtype=cuda.uint8, device="cuda")
    with pytest.raises(t213.T213Error) as e:
        t213.permute(dev, dims, perm, elem_bytes=4)
    assert e.value.status == 1


@pytest.mark.parametrize("shape,dims", [((4, 384, 512), (0, 2, 1)), ((2, 3, 5, 64, 48), (4, 2, 0, 3, 1)),
                                        ((30, 40, 50), (2, 1, 0)), ((7, 1, 9), (1, 2, 0)), ((16, 16), (1, 0))])
def test_torch_permute_(shape, dims):
    importlib.import_module("213transpose_b200.torch_op")
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randint(-2**31, 2**31 - 1, shape, generator=g, device="cuda", dtype=torch.int32)
    want = x.permute(dims).contiguous()
    y = torch.ops.t213.permute_(x, list(dims))
    torch.cuda.synchronize()
    assert y is x and x.shape == want.shape and x.is_contiguous()
    assert torch.equal(x.reshape(-1), want.reshape(-1))
