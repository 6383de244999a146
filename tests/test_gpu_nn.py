"""Tensor-core dense layers (tcgen05 MMA, TMEM accumulators) against a plain PyTorch FP32
reference of the same operation on the same BF16 operands.

Forward: y = W2 relu(W1 x + b1) + b2 + residual with x gathered from up to three sources;
the hidden activation is rounded to BF16 before the second product, as in the kernel.
Backward: dZ = (dY W2) * [h > 0] (BF16), dX = dZ W1, dW1^T = dZ^T X, dW2^T = dY^T H and the
bias sums.  The only differences allowed are FP32 summation order (and, for the forward
output, a BF16 rounding of the hidden tile that can fall either way)."""
import numpy as np
import pytest
import torch

from cabanadem_b200 import api, nn

pytestmark = pytest.mark.gpu


def _sources(kin, rows, gen, dev):
    """Input sources of a layer with `kin` features: edge-like rows gathered from node tables."""
    nodes = max(rows // 3, 7)
    bf = dict(device=dev, dtype=torch.bfloat16)
    if kin == 384:
        e = torch.randn(rows, 128, generator=gen).to(**bf)
        h = torch.randn(nodes, 128, generator=gen).to(**bf)
        ii = torch.randint(0, nodes, (rows,), generator=gen, dtype=torch.int32).to(dev)
        jj = torch.randint(0, nodes, (rows,), generator=gen, dtype=torch.int32).to(dev)
        return [(e, None), (h, ii), (h, jj)]
    if kin == 256:
        h = torch.randn(rows, 128, generator=gen).to(**bf)
        a = torch.randn(rows, 128, generator=gen).to(**bf)
        return [(h, None), (a, None)]
    x = torch.randn(rows, kin, generator=gen).to(**bf)
    return [(x, None)]


def _gather(srcs):
    return torch.cat([d.float() if i is None else d.float()[i.long()] for d, i in srcs], dim=1)


@pytest.mark.parametrize("kin,nout", nn.SHAPES)
@pytest.mark.parametrize("rows", [1000, 37, 148 * 128 + 200])
def test_mlp_forward_backward_matches_torch_fp32(kin, nout, rows):
    _check_layer(kin, nout, rows, resid_src0=False)


@pytest.mark.parametrize("kin", [256, 384])
def test_residual_from_source0(kin):
    """The message and update layers add their first input as residual (read from the staged tile)."""
    _check_layer(kin, 128, 2000, resid_src0=True)


def _check_layer(kin, nout, rows, resid_src0):
    dev = torch.device("cuda:0")
    ctx = api.Context(0)
    gen = torch.Generator().manual_seed(kin * 7 + nout + rows)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    with torch.cuda.stream(stream):
        m = nn.Mlp(kin, nout, dev, gen)
        m.b1.copy_(torch.randn(128, generator=gen) * 0.1)
        m.b2.copy_(torch.randn(nout, generator=gen) * 0.1)
        srcs = _sources(kin, rows, gen, dev)
        resid = srcs[0][0] if resid_src0 else torch.randn(rows, nout, generator=gen).to(dev, torch.bfloat16)
        out = torch.empty(rows, nout, device=dev, dtype=torch.bfloat16)
        out32 = torch.empty(rows, nout, device=dev, dtype=torch.float32)
        h1 = torch.empty(rows, 128, device=dev, dtype=torch.bfloat16)
        m.forward(ctx, rows, srcs, resid=resid, out=out, out_f32=out32, h1=h1)

        x = _gather(srcs)
        z = x @ m.w1t_bf.float().t() + m.b1
        h_ref = torch.relu(z).to(torch.bfloat16).float()
        y_ref = h_ref @ m.w2t_bf.float().t() + m.b2 + resid.float()
        # the hidden tile: equal up to a BF16 rounding of values that sit on a rounding edge
        dh = (h1.float() - h_ref).abs()
        assert (dh > 0).float().mean().item() < 1e-3
        assert dh.max().item() <= 1e-2 * max(h_ref.abs().max().item(), 1e-30)
        # the output from the kernel's own hidden tile: FP32 summation order only
        y_own = h1.float() @ m.w2t_bf.float().t() + m.b2 + resid.float()
        scale = y_own.abs().max().item()
        assert (out32 - y_own).abs().max().item() <= 1e-5 * scale
        assert (out32 - y_ref).abs().max().item() <= 1e-2 * scale
        assert (out.float() - out32).abs().max().item() <= 1e-2 * scale

        dy = torch.randn(rows, nout, generator=gen).to(dev, torch.bfloat16)
        dz1 = torch.empty(rows, 128, device=dev, dtype=torch.bfloat16)
        dx = torch.empty(rows, kin, device=dev, dtype=torch.float32)
        m.zero_grad()
        m.backward(ctx, rows, srcs, dy, h1, dz1, dx=dx)

        dz_ref = ((dy.float() @ m.w2t_bf.float()) * (h1.float() > 0)).to(torch.bfloat16).float()
        ddz = (dz1.float() - dz_ref).abs()
        assert ddz.max().item() <= 1e-2 * dz_ref.abs().max().item()
        dzk = dz1.float()
        dx_ref = dzk @ m.w1t_bf.float()
        assert (dx - dx_ref).abs().max().item() <= 1e-5 * dx_ref.abs().max().item()
        gw1t, gb1, gw2t, gb2 = m.grads
        r_gw1t = dzk.t() @ x
        r_gw2t = dy.float().t() @ h1.float()
        for got, ref in ((gw1t, r_gw1t), (gb1, dzk.sum(0)), (gw2t, r_gw2t), (gb2, dy.float().sum(0))):
            # sums over all rows: per-CTA partials added in block order vs torch's order
            assert (got - ref).abs().max().item() <= 1e-4 * ref.abs().max().item() + 1e-6
    assert nn.status(ctx) == 0
    ctx.close()


def test_backward_is_deterministic():
    dev = torch.device("cuda:0")
    ctx = api.Context(0)
    gen = torch.Generator().manual_seed(3)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    rows = 148 * 128 * 3 + 5
    with torch.cuda.stream(stream):
        m = nn.Mlp(384, 128, dev, gen)
        srcs = _sources(384, rows, gen, dev)
        h1 = torch.empty(rows, 128, device=dev, dtype=torch.bfloat16)
        m.forward(ctx, rows, srcs, h1=h1)
        dy = torch.randn(rows, 128, generator=gen).to(dev, torch.bfloat16)
        dz1 = torch.empty(rows, 128, device=dev, dtype=torch.bfloat16)
        got = []
        for _ in range(2):
            m.zero_grad()
            m.backward(ctx, rows, srcs, dy, h1, dz1)
            got.append([g.cpu().numpy().copy() for g in m.grads])
    for a, b in zip(*got):
        assert np.array_equal(a, b)
    ctx.close()


def test_wait_that_runs_out_is_reported_and_the_next_call_succeeds():
    """A bounded wait that runs out: with dem_nn_debug_waits(drop_mma=1) the kernels issue no
    MMA and no commit, so each block's wait on the completion barrier gives up after the poll
    limit (nothing is in flight, nothing faults).  The call reports DEM_ERR_TIMEOUT through
    dem_nn_status, and with the default bounds restored the same layer runs and matches the
    FP32 reference: the context stayed usable and no tensor memory was left allocated."""
    from cabanadem_b200 import _lib
    dev = torch.device("cuda:0")
    ctx = api.Context(0)
    gen = torch.Generator().manual_seed(11)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    rows = 148 * 128 + 77
    L = _lib.lib()
    with torch.cuda.stream(stream):
        m = nn.Mlp(128, 128, dev, gen)
        srcs = _sources(128, rows, gen, dev)
        out32 = torch.full((rows, 128), 7.0, device=dev, dtype=torch.float32)
        assert L.dem_nn_debug_waits(ctx.h, 1000, 1) == 0
        try:
            m.forward(ctx, rows, srcs, out_f32=out32)
            assert nn.status(ctx) == 0x020           # DEM_ERR_TIMEOUT
            assert bool((out32 == 7.0).all())        # no block got past its first wait
        finally:
            assert L.dem_nn_debug_waits(ctx.h, 0, 0) == 0
        m.forward(ctx, rows, srcs, out_f32=out32)
        assert nn.status(ctx) == 0
        x = _gather(srcs)
        h = torch.relu(x @ m.w1t_bf.float().t() + m.b1).to(torch.bfloat16).float()
        ref = h @ m.w2t_bf.float().t() + m.b2
        assert (out32 - ref).abs().max().item() <= 1e-2 * ref.abs().max().item()
    ctx.close()


def _edge_case(rows, gen, dev):
    bf = dict(device=dev, dtype=torch.bfloat16)
    nodes = max(rows // 3, 7)
    e = torch.randn(rows, 128, generator=gen).to(**bf)
    pq = (torch.randn(nodes, 256, generator=gen) * 0.5).to(**bf)
    recv = torch.randint(0, nodes, (rows,), generator=gen, dtype=torch.int32).to(dev)
    send = torch.randint(0, nodes, (rows,), generator=gen, dtype=torch.int32).to(dev)
    w1e_t = (torch.randn(128, 128, generator=gen) / 128 ** 0.5).to(**bf)
    w2t = (torch.randn(128, 128, generator=gen) / 128 ** 0.5).to(**bf)
    b1 = (torch.randn(128, generator=gen) * 0.1).to(dev)
    b2 = (torch.randn(128, generator=gen) * 0.1).to(dev)
    return e, pq, recv, send, w1e_t, b1, w2t, b2


@pytest.mark.parametrize("rows", [37, 1000, 2 * 148 * 128 + 200, 1_200_017])
def test_edge_layer_forms_match_torch_fp32(rows):
    """The factorised message layer, out = e + b2 + W2 relu(W1e e + b1 + P[recv] + Q[send]):
    the form whose e tiles come by tiled tensor copies (128-byte swizzle, one tile ahead) with
    the hidden tile in tensor memory as the second product's A operand, and the form staged by
    per-thread copies with the hidden tile in shared memory -- the same bits (outputs and hidden
    activations), and both equal to a PyTorch FP32 reference of the same operation on the same
    BF16 operands (hidden rounded to BF16 as in the kernels).  Row counts: a partial single tile,
    several tiles, more tiles than CTAs with a ragged last tile, and the 200k dam break's edge
    count."""
    dev = torch.device("cuda:0")
    ctx = api.Context(0)
    gen = torch.Generator().manual_seed(rows)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    with torch.cuda.stream(stream):
        e, pq, recv, send, w1e_t, b1, w2t, b2 = _edge_case(rows, gen, dev)
        outs = []
        for form in (0, 1):
            out = torch.full((rows, 128), 3.0, device=dev, dtype=torch.bfloat16)
            h1 = torch.full((rows, 128), 3.0, device=dev, dtype=torch.bfloat16)
            nn.edge_forward(ctx, e, pq, recv, send, w1e_t, b1, w2t, b2, out, h1, form=form)
            outs.append((out, h1))
        assert nn.status(ctx) == 0
        assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
        ef, pqf = e.float(), pq.float()
        z = ef @ w1e_t.float().t() + b1 + pqf[recv.long(), :128] + pqf[send.long(), 128:]
        h = torch.relu(z).to(torch.bfloat16).float()
        ref = h @ w2t.float().t() + b2 + ef
        got = outs[0][0].float()
        assert (got - ref).abs().max().item() <= 2e-2 * ref.abs().max().item()
        # hidden activations: equal up to a BF16 rounding of values on a rounding edge
        dh = (outs[0][1].float() - h).abs()
        assert dh.max().item() <= 2e-2 * h.abs().max().item()
        assert (dh > 0).float().mean().item() < 1e-3
    ctx.close()


def test_edge_layer_wait_that_runs_out_is_reported():
    """The tensor-copy form with dem_nn_debug_waits(drop_mma=1): the tile copies arrive, no MMA
    is issued, each block's wait on the product gives up; the call reports DEM_ERR_TIMEOUT and
    writes nothing, and with the default bounds restored the same call gives the staged form's
    bits."""
    from cabanadem_b200 import _lib
    dev = torch.device("cuda:0")
    ctx = api.Context(0)
    gen = torch.Generator().manual_seed(5)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    rows = 148 * 2 * 128 + 99
    L = _lib.lib()
    with torch.cuda.stream(stream):
        args = _edge_case(rows, gen, dev)
        out = torch.full((rows, 128), 7.0, device=dev, dtype=torch.bfloat16)
        assert L.dem_nn_debug_waits(ctx.h, 1000, 1) == 0
        try:
            nn.edge_forward(ctx, *args, out, None, form=0)
            assert nn.status(ctx) == 0x020           # DEM_ERR_TIMEOUT
            assert bool((out.float() == 7.0).all())
        finally:
            assert L.dem_nn_debug_waits(ctx.h, 0, 0) == 0
        ref = torch.empty_like(out)
        nn.edge_forward(ctx, *args, out, None, form=0)
        nn.edge_forward(ctx, *args, ref, None, form=1)
        assert nn.status(ctx) == 0
        assert torch.equal(out, ref)
    ctx.close()
