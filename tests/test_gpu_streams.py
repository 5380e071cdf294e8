"""Calls on one plan from two streams: plans whose device work uses internal
scratch (multi-dimensional mp and FP64 plans) order that work across streams,
so two calls issued back to back on different streams, without any host
synchronisation between them, give the results of the same calls made one
after another."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import mpfft_b200

    return mpfft_b200


def test_two_streams_rank2_mp_plan(M, orc):
    import torch

    O = orc
    dims, p, batch = (32, 64), 256, 16
    plan = M.MpPlanND(dims, p)
    n = plan.n
    ins = []
    for seed in (1, 2):
        xr, xi = O.mp_pair(n * batch, p)
        O.fill_uniform(xr, xi, seed)
        host = np.zeros(plan.words(batch), dtype=np.uint32)
        exps = np.zeros(batch, dtype=np.int64)
        plan.pack(batch, xr.ptr, xi.ptr, host.ctypes.data, exps.ctypes.data)
        ins.append(torch.from_numpy(host.view(np.int32)).cuda())
    # sequential reference results
    ref = []
    for d_in in ins:
        out = torch.empty_like(d_in)
        plan.execute_device(batch, d_in.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        ref.append(out.cpu())
    # both calls in flight on two streams
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    outs = [torch.full_like(ins[0], -1), torch.full_like(ins[1], -1)]
    torch.cuda.synchronize()  # the fills ran on the current stream
    for _ in range(3):
        plan.execute_device(batch, ins[0].data_ptr(), outs[0].data_ptr(), s1.cuda_stream)
        plan.execute_device(batch, ins[1].data_ptr(), outs[1].data_ptr(), s2.cuda_stream)
    torch.cuda.synchronize()
    for got, want in zip(outs, ref):
        assert torch.equal(got.cpu(), want)


def test_two_streams_rank2_fp64_plan(M):
    import torch

    dims, batch = (64, 128), 8
    plan = M.DPlanND(dims)
    n = dims[0] * dims[1]
    g = torch.Generator().manual_seed(3)
    ins = [torch.rand(2 * batch * n, dtype=torch.float64, generator=g).cuda() for _ in range(2)]
    ref = []
    for d_in in ins:
        out = torch.empty_like(d_in)
        plan.execute_device(batch, d_in.data_ptr(), out.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        ref.append(out.cpu())
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    outs = [torch.empty_like(ins[0]), torch.empty_like(ins[1])]
    torch.cuda.synchronize()
    for _ in range(3):
        plan.execute_device(batch, ins[0].data_ptr(), outs[0].data_ptr(), stream=s1.cuda_stream)
        plan.execute_device(batch, ins[1].data_ptr(), outs[1].data_ptr(), stream=s2.cuda_stream)
    torch.cuda.synchronize()
    for got, want in zip(outs, ref):
        assert torch.equal(got.cpu(), want)


def test_device_calls_replayed_and_inside_a_callers_graph(M):
    """A one-signal device-layout call replays its own CUDA graph from the
    second call on, and inside a graph the caller is capturing it launches
    its kernels into that capture instead: all give the first call's output
    bit for bit."""
    import torch

    from mpfft_b200.mparray import synthetic_planes

    n = 1024
    plan = M.MpPlan(n, 1024)
    host = synthetic_planes(n, plan.limbs, plan.frac_bits, 1, seed=9)
    d_in = torch.from_numpy(host.view(np.int32)).cuda()
    outs = [torch.empty_like(d_in) for _ in range(3)]
    s = torch.cuda.current_stream().cuda_stream
    for _ in range(3):  # direct, then captured and replayed
        plan.execute_device(1, d_in.data_ptr(), outs[0].data_ptr(), s)
    plan.execute_device(1, d_in.data_ptr(), outs[1].data_ptr(), s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        with torch.cuda.graph(g, stream=side):
            plan.execute_device(1, d_in.data_ptr(), outs[2].data_ptr(), side.cuda_stream)
    g.replay()
    torch.cuda.synchronize()
    ref = outs[0].cpu().numpy()
    assert np.array_equal(outs[1].cpu().numpy(), ref)
    assert np.array_equal(outs[2].cpu().numpy(), ref)
