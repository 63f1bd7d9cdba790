"""Mixed batches (zlfft_mixed_*): transforms of many orders, kinds and
operations in one call, with per-transform device pointers.

Every transform of a mixed batch must give the same bits as the same
transform run alone through zlfft_exec_device (the kernels' arithmetic is the
same), and in FP32 the same bits as the oracle; all three schedules (per-order
loop, persistent launch, CUDA graph replay) must agree.
"""
import ctypes

import numpy as np
import pytest

import zldsp_fft_b200 as Z
from tests import gpu_util as G

pytestmark = pytest.mark.gpu

ALIGN = 64  # bytes between transforms in the packed test buffers


class Packed:
    """Transforms placed at shuffled, aligned offsets of one input and one
    output buffer, so the batch's pointers follow no stride."""

    def __init__(self, rng, specs):
        import torch
        self.specs = specs
        self.x = []
        in_sz, out_sz = [], []
        for s in specs:
            kind, order, op, prec = s
            n = 1 << order
            rdt = np.float32 if prec == Z.F32 else np.float64
            cdt = np.complex64 if prec == Z.F32 else np.complex128
            if kind == Z.C2C:
                x = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(cdt)
                o = n * x.itemsize
            elif op == Z.BACKWARD:
                nb = n // 2 + 1
                x = (rng.uniform(-1, 1, nb) + 1j * rng.uniform(-1, 1, nb)).astype(cdt)
                x[0] = x[0].real
                x[-1] = x[-1].real
                o = n * np.dtype(rdt).itemsize
            else:
                x = rng.uniform(-1, 1, n).astype(rdt)
                nb = n // 2 + 1
                o = nb * (np.dtype(cdt).itemsize if op == Z.FORWARD else np.dtype(rdt).itemsize)
            self.x.append(x)
            in_sz.append(x.nbytes)
            out_sz.append(o)
        up = lambda v: (v + ALIGN - 1) // ALIGN * ALIGN
        self.in_off = self._place(rng, [up(v) for v in in_sz])
        self.out_off = self._place(rng, [up(v) for v in out_sz])
        self.out_sz = out_sz
        self.tin = torch.zeros(max(1, sum(up(v) for v in in_sz)), dtype=torch.uint8, device="cuda")
        self.tout = torch.zeros(max(1, sum(up(v) for v in out_sz)), dtype=torch.uint8, device="cuda")
        self.upload()

    @staticmethod
    def _place(rng, sizes):
        order = rng.permutation(len(sizes))
        off, pos = [0] * len(sizes), 0
        for i in order:
            off[i] = pos
            pos += sizes[i]
        return off

    def upload(self):
        import torch
        host = np.zeros(self.tin.numel(), dtype=np.uint8)
        for x, o in zip(self.x, self.in_off):
            b = x.view(np.uint8)
            host[o:o + b.size] = b
        self.tin.copy_(torch.from_numpy(host))

    def descs(self, in_place=()):
        base_i, base_o = self.tin.data_ptr(), self.tout.data_ptr()
        out = []
        for i, (kind, order, op, prec) in enumerate(self.specs):
            ip = base_i + self.in_off[i]
            op_ptr = ip if i in in_place else base_o + self.out_off[i]
            out.append((kind, order, op, ip, op_ptr, prec))
        return out

    def results(self, in_place=()):
        bi = self.tin.cpu().numpy()
        bo = self.tout.cpu().numpy()
        res = []
        for i, (kind, order, op, prec) in enumerate(self.specs):
            rdt = np.float32 if prec == Z.F32 else np.float64
            cdt = np.complex64 if prec == Z.F32 else np.complex128
            src, off = (bi, self.in_off[i]) if i in in_place else (bo, self.out_off[i])
            raw = src[off:off + self.out_sz[i]].copy()
            complex_out = kind == Z.C2C or op == Z.FORWARD
            res.append(raw.view(cdt) if complex_out else raw.view(rdt))
        return res


def _single(spec, x):
    """The same transform alone through zlfft_exec_device."""
    kind, order, op, prec = spec
    dt = np.float32 if prec == Z.F32 else np.float64
    plan = Z.Plan(kind, order, dt)
    if kind == Z.C2C:
        return G.run_c2c(plan, x[None], op == Z.FORWARD)[0]
    if op == Z.BACKWARD:
        return G.run_c2r(plan, x[None])[0]
    return G.run_r2c(plan, x[None], Z.AOS, sqr_mag=(op == Z.FORWARD_SQR_MAG))[0]


def _oracle(oracle, spec, x):
    kind, order, op, prec = spec
    if kind == Z.C2C:
        return oracle.cfft_port(x[None], op == Z.FORWARD)[0]
    if op == Z.BACKWARD:
        return oracle.rfft_backward_port(x[None])[0]
    return oracle.rfft_forward_port(x[None], sqr_mag=(op == Z.FORWARD_SQR_MAG))[0]


def _run(pk, schedule, descs=None, in_place=()):
    import torch
    pk.tout.zero_()
    mb = Z.MixedBatch(descs or pk.descs(in_place))
    mb.run(schedule)
    torch.cuda.synchronize()
    assert mb.device_status() == 0
    return mb, pk.results(in_place)


def test_mixed_cfg_like_batch_all_schedules(oracle):
    """A seeded batch shaped like the mixed-order workload (orders 6..16, half
    CFFT forward, half RFFT forward, AoS, uniform [-1, 1) data): every schedule
    gives the oracle's bits for every transform."""
    import torch
    rng = np.random.default_rng(1004)
    specs = []
    for _ in range(240):
        order = int(rng.integers(6, 17))
        specs.append((Z.C2C, order, Z.FORWARD, Z.F32) if rng.random() < 0.5 else (Z.R2C, order, Z.FORWARD, Z.F32))
    pk = Packed(rng, specs)
    expect = [_oracle(oracle, s, x) for s, x in zip(specs, pk.x)]
    outs = {}
    for sched in (Z.SCHED_PER_ORDER, Z.SCHED_PERSISTENT, Z.SCHED_GRAPH):
        mb, res = _run(pk, sched)
        outs[sched] = res
        bad = [i for i, (y, e) in enumerate(zip(res, expect)) if not np.array_equal(y, e)]
        assert not bad, (sched, [specs[i] for i in bad[:5]], len(bad))
        assert mb.take_launch_count() > 0
    # the persistent schedule needs fewer launches than the per-order loop
    mb = Z.MixedBatch(pk.descs())
    mb.run(Z.SCHED_PER_ORDER)
    n_loop = mb.take_launch_count()
    mb.run(Z.SCHED_PERSISTENT)
    n_pers = mb.take_launch_count()
    mb.run(Z.SCHED_GRAPH)
    n_graph = mb.take_launch_count()
    torch.cuda.synchronize()
    assert n_pers < n_loop and n_graph == n_pers
    for i, (s, x) in enumerate(zip(specs, pk.x)):
        if i % 40 == 0:  # accuracy against FP64 as well
            ref = oracle.cfft_fp64(x[None]) if s[0] == Z.C2C else oracle.rfft_fp64(x[None])
            assert oracle.rel_l2(outs[Z.SCHED_GRAPH][i][None], ref).max() <= oracle.tolerance(s[1], "f32")


def test_mixed_every_operation_order_and_precision(oracle):
    """Every kind/operation at edge and pass-boundary orders (0, 1, 2, 11, 12,
    13, 14, 15), FP32 and FP64 in one batch: identical to the same transform
    run alone, and within the FP64 oracle tolerance (FP32: the oracle's bits)."""
    rng = np.random.default_rng(77)
    specs = []
    for prec in (Z.F32, Z.F64):
        for order in (0, 1, 2, 3, 5, 11, 12, 13, 14, 15):
            specs.append((Z.C2C, order, Z.FORWARD, prec))
            specs.append((Z.C2C, order, Z.BACKWARD, prec))
        for order in (1, 2, 3, 6, 12, 13, 14, 15, 16):
            for op in (Z.FORWARD, Z.FORWARD_SQR_MAG, Z.BACKWARD):
                specs.append((Z.R2C, order, op, prec))
    specs = specs * 2  # two transforms per group
    pk = Packed(rng, specs)
    for sched in (Z.SCHED_PERSISTENT, Z.SCHED_PER_ORDER):
        _, res = _run(pk, sched)
        for i, (s, x, y) in enumerate(zip(specs, pk.x, res)):
            alone = _single(s, x)
            assert np.array_equal(y, alone), (sched, s)
            if s[3] == Z.F32:
                assert np.array_equal(y, _oracle(oracle, s, x)), (sched, s)
            else:
                kind, order, op, _ = s
                if kind == Z.C2C:
                    ref = oracle.cfft_fp64(x[None], op == Z.FORWARD)
                elif op == Z.BACKWARD:
                    ref = oracle.rfft_backward_fp64(x[None])
                else:
                    ref = oracle.rfft_fp64(x[None])
                    if op == Z.FORWARD_SQR_MAG:
                        ref = np.abs(ref) ** 2
                assert oracle.rel_l2(y[None], ref).max() <= oracle.tolerance(max(order, 1), "f64"), s


def test_mixed_in_place_and_graph_replay_follows_new_data(oracle):
    """In-place CFFT descriptors; a graph replayed after the inputs change
    computes on the new data (the graph records pointers, not values)."""
    import torch
    rng = np.random.default_rng(5)
    specs = [(Z.C2C, int(o), Z.FORWARD, Z.F32) for o in rng.integers(6, 15, 60)]
    specs += [(Z.R2C, int(o), Z.FORWARD, Z.F32) for o in rng.integers(6, 15, 60)]
    in_place = set(range(0, 60, 2))
    pk = Packed(rng, specs)
    mb = Z.MixedBatch(pk.descs(in_place))
    for rep in range(2):
        if rep:
            pk.x = [(-2 * x).astype(x.dtype) for x in pk.x]
        pk.upload()
        pk.tout.zero_()
        mb.run(Z.SCHED_GRAPH)
        torch.cuda.synchronize()
        res = pk.results(in_place)
        for s, x, y in zip(specs, pk.x, res):
            assert np.array_equal(y, _oracle(oracle, s, x)), (rep, s)
    assert mb.device_status() == 0


def test_exec_mixed_device_one_shot(oracle):
    """zlfft_exec_mixed_device: create, run on the stream, synchronise, destroy."""
    rng = np.random.default_rng(9)
    specs = [(Z.C2C, 8, Z.FORWARD, Z.F32), (Z.R2C, 10, Z.FORWARD_SQR_MAG, Z.F32), (Z.C2C, 14, Z.BACKWARD, Z.F32)]
    pk = Packed(rng, specs)
    arr = (Z._capi.Desc * len(specs))(*[Z._capi.Desc(k, p, o, op, i, out) for k, o, op, i, out, p in pk.descs()])
    assert Z._capi.lib().zlfft_exec_mixed_device(arr, len(specs), None) == 0, Z._capi.last_error()
    for s, x, y in zip(specs, pk.x, pk.results()):
        assert np.array_equal(y, _oracle(oracle, s, x)), s
    # an empty batch is a no-op
    assert Z._capi.lib().zlfft_exec_mixed_device(None, 0, None) == 0


def test_mixed_orders_6_to_20_all_schedules(oracle):
    """A batch over the whole range of the mixed-order target, 2^6 to 2^20,
    CFFT forward/backward and RFFT forward/forward_sqr_mag/backward, FP32:
    both persistent classes (complex orders 2..11 and 12..13), the order-14
    tile and the multi-pass pipelines (up to 2^20, several transforms per
    order). Every schedule gives the oracle's bits for every transform."""
    rng = np.random.default_rng(2020)
    specs = []
    for order in range(6, 21):
        reps = 6 if order <= 13 else (3 if order <= 17 else 2)
        for _ in range(reps):
            specs.append((Z.C2C, order, Z.FORWARD, Z.F32))
            specs.append((Z.C2C, order, Z.BACKWARD, Z.F32))
            specs.append((Z.R2C, order, (Z.FORWARD, Z.FORWARD_SQR_MAG, Z.BACKWARD)[int(rng.integers(3))], Z.F32))
    order_perm = rng.permutation(len(specs))
    specs = [specs[i] for i in order_perm]
    pk = Packed(rng, specs)
    expect = [_oracle(oracle, s, x) for s, x in zip(specs, pk.x)]
    for sched in (Z.SCHED_PER_ORDER, Z.SCHED_PERSISTENT, Z.SCHED_GRAPH):
        _, res = _run(pk, sched)
        bad = [i for i, (y, e) in enumerate(zip(res, expect)) if not np.array_equal(y, e)]
        assert not bad, (sched, [specs[i] for i in bad[:5]], len(bad))
