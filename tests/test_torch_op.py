"""The PyTorch binding torch.ops.t213.transpose_: registration, shape and
refusals on the host; values on the GPU against torch's own out-of-place
transpose (bit-exact)."""
import importlib

import pytest
import torch

op = importlib.import_module("213transpose_b200.torch_op")


def test_registered_and_meta_shape():
    x = torch.empty(5, 3, 4, device="meta")
    y = torch.ops.t213.transpose_(x)
    assert y is x and tuple(x.shape) == (5, 4, 3) and x.is_contiguous()


def test_permute_meta_shape():
    x = torch.empty(2, 3, 4, 5, device="meta")
    torch.ops.t213.permute_(x, [3, 1, 0, 2])
    assert tuple(x.shape) == (5, 3, 2, 4) and x.is_contiguous()
    with pytest.raises(Exception):
        torch.ops.t213.permute_(torch.empty(2, 3, device="meta"), [0, 0])


def test_refuses_cpu_tensors():
    with pytest.raises(RuntimeError):
        torch.ops.t213.transpose_(torch.zeros(2, 3, 4))


@pytest.mark.parametrize("dims", [(0, 1), (0, 2), (-3, -1)])
def test_refuses_other_dims(dims):
    with pytest.raises(Exception):
        torch.ops.t213.transpose_(torch.empty(2, 3, 4, device="meta"), *dims)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,dtype", [((4, 384, 512), torch.float32), ((2, 6151, 7919), torch.float64),
                                         ((3, 97, 300), torch.int32), ((2, 3, 5, 64, 48), torch.float16),
                                         ((1000, 999), torch.float32), ((0, 7, 5), torch.float32),
                                         ((8, 1, 9), torch.int64)])
def test_values_match_torch(shape, dtype):
    g = torch.Generator(device="cuda").manual_seed(0)
    if dtype.is_floating_point:
        x = torch.rand(shape, generator=g, device="cuda").to(dtype)
    else:
        x = torch.randint(-1000, 1000, shape, generator=g, device="cuda", dtype=dtype)
    want = x.transpose(-2, -1).contiguous()
    ptr = x.data_ptr()
    y = torch.ops.t213.transpose_(x)
    torch.cuda.synchronize()
    assert y is x and x.data_ptr() == ptr and x.is_contiguous()
    assert x.shape == want.shape
    # byte views of the flattened tensors (size-1 and empty dimensions may
    # carry any stride)
    assert torch.equal(x.reshape(-1).view(torch.uint8), want.reshape(-1).view(torch.uint8))


@pytest.mark.gpu
def test_refuses_non_contiguous():
    x = torch.zeros(4, 6, 8, device="cuda").transpose(1, 2)
    with pytest.raises(ValueError):
        torch.ops.t213.transpose_(x)
