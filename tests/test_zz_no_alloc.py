"""hpcg_b200_dot_noalloc, the dot product for callers that cannot allocate
device memory: their own allocator owns the GPU's memory, or they call from a
place where a cudaMalloc (which also synchronises the device) is not allowed.

It is checked through the C ABI against the allocating entry point
hpcg_b200_dot and against the correctly rounded sum of the products
(math.fsum), within the dot-product tolerance of the other GPU tests (relative
1e-13), on two calls in a row, and its size limit and pointer checks are
exercised: host memory and another GPU's memory are refused before anything
runs. This file is named to be collected last."""
import ctypes as C
import math

import pytest

pytestmark = pytest.mark.gpu

MAX_N = 268435456  # HPCG_B200_DOT_NOALLOC_MAX_N


def test_noalloc_dot_matches_allocating_dot_on_two_calls(binding):
    import torch
    lib = binding.lib()
    for call, n in enumerate((1 << 20, 3 * 4096 + 17)):
        g = torch.Generator(device="cuda").manual_seed(100 + call)
        x = torch.rand(n, dtype=torch.float64, device="cuda", generator=g)
        y = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) - 0.5
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        status = lib.hpcg_b200_dot_noalloc(n, x.data_ptr(), y.data_ptr(), out.data_ptr(), None)
        assert status == 0, binding.last_error()
        torch.cuda.synchronize()
        if call == 1:  # after the first call's set-up: nothing is allocated
            assert torch.cuda.mem_get_info()[0] == free_before
        got = out.item()
        ref = binding.ComputeDotProduct(n, x, y)
        exact = math.fsum((x * y).cpu().numpy())
        bound = 1e-13 * max(abs(exact), float((x * y).abs().sum()) * 1e-3)
        assert abs(got - ref) <= bound, (got, ref)
        assert abs(got - exact) <= bound, (got, exact)


def test_noalloc_dot_limits(binding):
    import torch
    lib = binding.lib()
    x = torch.ones(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert lib.hpcg_b200_dot_noalloc(MAX_N + 1, x.data_ptr(), x.data_ptr(), out.data_ptr(), None) == binding.ERR_ARG
    assert "outside" in binding.last_error()
    host = (C.c_double * 8)()
    assert lib.hpcg_b200_dot_noalloc(8, C.addressof(host), x.data_ptr(), out.data_ptr(), None) == binding.ERR_ARG
    assert lib.hpcg_b200_dot_noalloc(0, x.data_ptr(), x.data_ptr(), out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert out.item() == 0.0
    assert lib.hpcg_b200_dot_noalloc(8, x.data_ptr(), x.data_ptr(), out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert out.item() == 8.0


def test_noalloc_dot_refuses_another_gpus_memory(binding):
    """A pointer to a second GPU's memory passed while the first is current is
    refused with HPCG_B200_ERR_ARG (no kernel runs). Needs two visible GPUs."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("one GPU visible")
    lib = binding.lib()
    torch.cuda.set_device(0)
    x = torch.ones(8, dtype=torch.float64, device="cuda:0")
    other = torch.ones(8, dtype=torch.float64, device="cuda:1")
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    assert lib.hpcg_b200_dot_noalloc(8, x.data_ptr(), other.data_ptr(), out.data_ptr(), None) == binding.ERR_ARG
    assert "GPU 1" in binding.last_error()
