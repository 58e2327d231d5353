"""t-slab domain decomposition of the dslash across ranks.

The lattice is split along t into ``nodes_t`` slabs, one per rank (as the
reference's GJP.Nodes(3) with its QMP halo exchange in wilson_dslash_vec,
d_op_wilson/qmp/wilson_dslash_vec.C:184-278).  Each rank's ``Lattice`` holds
its slab (node_sites with Lt / nodes_t t-slices, an even number) and its
links; ``set_t_partition`` marks it.  One decomposed dslash is

    pack(D, inp, cb, dag, faces)          # the input's two t faces
    exchange_faces(faces)                 # to the neighbouring ranks
    dslash(D, out, inp, cb, dag, faces)   # the hop, reading the halos

or, with the exchange overlapped by the interior t-slices' hop,

    pack(D, inp, cb, dag, faces)
    dslash_interior(D, out, inp, cb, dag)          # enqueued, not waited for
    exchange_faces(faces)
    dslash_boundary(D, out, inp, cb, dag, faces)   # the two end t-slices

The faces are device buffers (torch uint8 tensors on the rank's GPU, only
plumbing); ``exchange_faces`` moves them with torch.distributed
point-to-point operations (NCCL between GPUs).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch
import torch.distributed as dist

from . import _abi as A
from ._abi import check, lib


class DeviceField:
    """a fermion field resident on the device (cpsgpu_field), one
    preconditioned checkerboard of the operator, in precision prec"""

    def __init__(self, D, prec=A.DOUBLE, nrhs=1):
        self.D, self.prec, self.nrhs = D, prec, nrhs
        self._h = C.c_void_p()
        check(lib().cpsgpu_field_create(D._h, prec, nrhs, C.byref(self._h)))

    def upload(self, host):
        host = np.ascontiguousarray(host, dtype=np.float64)
        if host.size != self.D.f_size * self.nrhs:
            raise ValueError("host vector of the wrong size")
        check(lib().cpsgpu_field_upload(self._h, host.ctypes.data_as(A._dp)))

    def download(self):
        out = np.empty(self.D.f_size * self.nrhs)
        check(lib().cpsgpu_field_download(self._h, out.ctypes.data_as(A._dp)))
        return out

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().cpsgpu_field_destroy(self._h)
            self._h = C.c_void_p()


def set_t_partition(lat, nodes_t: int, coor_t: int) -> None:
    """mark lat as slab coor_t of nodes_t along t"""
    check(lib().cpsgpu_lattice_set_t_partition(lat._h, nodes_t, coor_t))


class Faces:
    """the four face buffers of one rank: what it sends (to_prev, to_next)
    and what it receives (from_next, from_prev)"""

    def __init__(self, D, prec=A.DOUBLE, nrhs=1, device=None):
        n = C.c_size_t()
        check(lib().cpsgpu_dd_face_bytes(D._h, prec, nrhs, C.byref(n)))
        dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        mk = lambda: torch.empty(n.value, dtype=torch.uint8, device=dev)
        self.to_prev, self.to_next, self.from_next, self.from_prev = mk(), mk(), mk(), mk()


def pack(D, inp: DeviceField, cb: int, dag: int, faces: Faces) -> None:
    """pack the t faces of inp: (1 - sdag g_t) psi of the first t-slice
    (to_prev) and U_t^dagger (1 + sdag g_t) psi of the last (to_next)"""
    check(lib().cpsgpu_dslash_dd_pack(D._h, inp._h, cb, dag, C.c_void_p(faces.to_prev.data_ptr()),
                                      C.c_void_p(faces.to_next.data_ptr())))


def dslash(D, out: DeviceField, inp: DeviceField, cb: int, dag: int, faces: Faces) -> None:
    """the hop of inp into out, the t neighbours across the slab ends from
    the received faces"""
    check(lib().cpsgpu_dslash_dd(D._h, out._h, inp._h, cb, dag, C.c_void_p(faces.from_next.data_ptr()),
                                 C.c_void_p(faces.from_prev.data_ptr())))


def dslash_interior(D, out: DeviceField, inp: DeviceField, cb: int, dag: int) -> None:
    """the hop into the slab's interior t-slices (no halo read), enqueued
    on the library's stream: the device computes it while the faces move"""
    check(lib().cpsgpu_dslash_dd_interior(D._h, out._h, inp._h, cb, dag))


def dslash_boundary(D, out: DeviceField, inp: DeviceField, cb: int, dag: int, faces: Faces) -> None:
    """the hop into the slab's first and last t-slices from the received
    faces; returns when the interior part has finished too"""
    check(lib().cpsgpu_dslash_dd_boundary(D._h, out._h, inp._h, cb, dag, C.c_void_p(faces.from_next.data_ptr()),
                                          C.c_void_p(faces.from_prev.data_ptr())))


# point-to-point tags of the two face streams
TAG_TO_PREV, TAG_TO_NEXT = 17, 18


def exchange_faces(faces: Faces, group=None) -> None:
    """to_prev -> the previous rank's from_next, to_next -> the next rank's
    from_prev, over the periodic ring of the group's ranks"""
    rank, size = dist.get_rank(group), dist.get_world_size(group)
    if size == 1:
        faces.from_next.copy_(faces.to_prev)
        faces.from_prev.copy_(faces.to_next)
        return
    prev, nxt = (rank - 1) % size, (rank + 1) % size
    if group is not None:
        prev, nxt = dist.get_global_rank(group, prev), dist.get_global_rank(group, nxt)
    ops = [dist.P2POp(dist.isend, faces.to_prev, prev, group, TAG_TO_PREV),
           dist.P2POp(dist.irecv, faces.from_next, nxt, group, TAG_TO_PREV),
           dist.P2POp(dist.isend, faces.to_next, nxt, group, TAG_TO_NEXT),
           dist.P2POp(dist.irecv, faces.from_prev, prev, group, TAG_TO_NEXT)]
    for r in dist.batch_isend_irecv(ops):
        r.wait()


# ---- the decomposed operator and CG ----

def axpby(out: DeviceField, a: float, x: DeviceField, y: DeviceField) -> None:
    """out = a x + y (FP64 fields)"""
    check(lib().cpsgpu_field_axpby(out._h, a, x._h, y._h))


def axpby_device(out: DeviceField, a: torch.Tensor, scale: float, x: DeviceField, y: DeviceField) -> None:
    """out = (scale * a) x + y (FP64 fields), a a float64 device tensor read
    on the device; only enqueued"""
    check(lib().cpsgpu_field_axpby_device(out._h, C.c_void_p(a.data_ptr()), scale, x._h, y._h))


def dot_device(a: DeviceField, b: DeviceField, out: torch.Tensor) -> None:
    """out[0], out[1] = this rank's <a, b> (re, im), out a float64 device
    tensor of (at least) two elements; only enqueued"""
    check(lib().cpsgpu_field_dot_device(a._h, b._h, C.c_void_p(out.data_ptr())))


def set_stream(lat, stream) -> None:
    """every launch for lat on the CUDA stream `stream` (a created
    torch.cuda.Stream, not the legacy default stream, whose handle is null),
    the pack / dslash / axpby calls of the decomposition only enqueued; None
    restores the library's own stream"""
    if stream is not None and not stream.cuda_stream:
        raise ValueError("the legacy default stream cannot be the lattice's stream: use a created stream")
    check(lib().cpsgpu_lattice_set_stream(lat._h, C.c_void_p(stream.cuda_stream) if stream is not None else None))


def local_dot(a: DeviceField, b: DeviceField) -> complex:
    """this rank's part of <a, b> = sum conj(a) b (FP64 fields)"""
    re, im = C.c_double(), C.c_double()
    check(lib().cpsgpu_field_dot(a._h, b._h, C.byref(re), C.byref(im)))
    return complex(re.value, im.value)


class InProcessRing:
    """every slab of the lattice in this process: faces move between the
    slabs by device copies, a global sum is the sum over the slabs"""

    def exchange(self, faces, sync=True):
        n = len(faces)
        for r in range(n):
            faces[r].from_next.copy_(faces[(r + 1) % n].to_prev)
            faces[r].from_prev.copy_(faces[(r - 1) % n].to_next)
        # torch's stream only: an interior hop on the library's stream runs on
        if sync:
            torch.cuda.current_stream().synchronize()

    def allreduce(self, v: complex) -> complex:
        return v

    def allreduce_device(self, t: torch.Tensor) -> None:
        """t summed over the ranks in place (one rank here)"""


class _HostFaces:
    """host copies of a rank's faces, for a backend without device
    point-to-point (gloo)"""

    def __init__(self, f: Faces):
        self.to_prev, self.to_next = f.to_prev.cpu(), f.to_next.cpu()
        self.from_next, self.from_prev = torch.empty_like(self.to_prev), torch.empty_like(self.to_next)


class DistRing:
    """one slab per rank of a torch.distributed group: faces by
    point-to-point operations, global sums by all_reduce (the reference's
    glb_sum).  With NCCL the device faces move directly; with gloo they
    are staged through host memory."""

    def __init__(self, group=None):
        self.group = group

    def exchange(self, faces, sync=True):
        if len(faces) != 1:
            raise ValueError("one slab per rank")
        f = faces[0]
        if not sync:
            # the device-resident solver: NCCL point-to-point on the current
            # stream, ordered with the library's launches on the same stream
            if dist.get_backend(self.group) != "nccl":
                raise RuntimeError("a device-resident exchange needs the NCCL backend")
            exchange_faces(f, self.group)
            return
        # the pack call returned after its kernels, so the faces are ready;
        # only torch's stream is waited for, not an interior hop in flight
        # on the library's stream
        if dist.get_backend(self.group) == "nccl" or not f.to_prev.is_cuda:
            exchange_faces(f, self.group)
        else:
            h = _HostFaces(f)
            exchange_faces(h, self.group)
            f.from_next.copy_(h.from_next)
            f.from_prev.copy_(h.from_prev)
        if f.to_prev.is_cuda:
            torch.cuda.current_stream().synchronize()

    def allreduce_device(self, t: torch.Tensor) -> None:
        """t summed over the ranks in place, on the current stream (NCCL)"""
        if dist.get_backend(self.group) != "nccl":
            raise RuntimeError("a device-resident all-reduce needs the NCCL backend")
        dist.all_reduce(t, group=self.group)

    def allreduce(self, v: complex) -> complex:
        # NCCL reduces device tensors only; gloo (the CPU tests) host tensors
        on_gpu = dist.get_backend(self.group) == "nccl"
        dev = torch.device("cuda", torch.cuda.current_device()) if on_gpu else torch.device("cpu")
        t = torch.tensor([v.real, v.imag], dtype=torch.float64, device=dev)
        dist.all_reduce(t, group=self.group)
        return complex(t[0].item(), t[1].item())


class DDOperator:
    """MatPc / MatPcDagMatPc of a Wilson or DWF operator over t slabs
    (wilson_m.C:49-93, dwf_m.C:31-63: out = in - kappa^2 D_cb0 D_cb1 in):
    ops holds this process's slabs' DiracOps, ring moves faces and adds
    the ranks' parts of a dot product"""

    def __init__(self, ops, ring, overlap=True):
        self.ops, self.ring, self.overlap = list(ops), ring, overlap
        self.faces = [Faces(D) for D in self.ops]
        self.t1 = self.field()
        self.t2 = self.field()

    def field(self):
        return [DeviceField(D) for D in self.ops]

    def dslash(self, out, inp, cb, dag):
        for D, i, f in zip(self.ops, inp, self.faces):
            pack(D, i, cb, dag, f)
        if self.overlap:
            # interior t-slices on the device while the faces move
            for D, o, i in zip(self.ops, out, inp):
                dslash_interior(D, o, i, cb, dag)
            self.ring.exchange(self.faces)
            for D, o, i, f in zip(self.ops, out, inp, self.faces):
                dslash_boundary(D, o, i, cb, dag, f)
            return
        self.ring.exchange(self.faces)
        for D, o, i, f in zip(self.ops, out, inp, self.faces):
            dslash(D, o, i, cb, dag, f)

    def dot(self, a, b) -> complex:
        return self.ring.allreduce(sum((local_dot(x, y) for x, y in zip(a, b)), 0j))

    @staticmethod
    def axpby(out, a: float, x, y) -> None:
        axpby(out, a, x, y)

    def matpc(self, out, inp, dag=0):
        self.dslash(self.t1, inp, 1, dag)
        self.dslash(out, self.t1, 0, dag)
        for D, o, i in zip(self.ops, out, inp):
            axpby(o, -D.kappa * D.kappa, o, i)

    def mdagm(self, out, inp) -> float:
        """out = MatPcDag MatPc inp; returns |MatPc inp|^2"""
        self.matpc(self.t2, inp, 0)
        pap = self.dot(self.t2, self.t2).real
        self.matpc(out, self.t2, 1)
        return pap


def cg(op: DDOperator, x, b, stop_rsd=1e-8, max_num_iter=10000):
    """CG on MatPcDagMatPc over the slabs (the recurrences of InvCgShift,
    inv_cg.C:84-448: stop when |r|^2 <= stop_rsd^2 |b|^2), x the initial
    guess in, solution out; returns (iterations + 1 as the reference
    counts, true residual |b - A x| / |b|).  The host drives it: every
    global sum is a ring all-reduce.  op provides field(), dot(a, b) (the
    global sum of the slabs' dot products), mdagm(out, inp) and
    axpby(out, a, x, y) on one slab's field."""
    r, p, ap = op.field(), op.field(), op.field()
    bb = op.dot(b, b).real
    op.mdagm(ap, x)
    for ri, bi, ai in zip(r, b, ap):
        op.axpby(ri, -1.0, ai, bi)
    for pi, ri in zip(p, r):
        op.axpby(pi, 0.0, ri, ri)  # p = r
    rr = op.dot(r, r).real
    stop = stop_rsd * stop_rsd * bb
    k = 0
    while k < max_num_iter - 1 and rr > stop:
        pap = op.mdagm(ap, p)
        alpha = rr / pap
        for xi, pi in zip(x, p):
            op.axpby(xi, alpha, pi, xi)
        for ri, ai in zip(r, ap):
            op.axpby(ri, -alpha, ai, ri)
        rr_new = op.dot(r, r).real
        beta, rr = rr_new / rr, rr_new
        for pi, ri in zip(p, r):
            op.axpby(pi, beta, pi, ri)
        k += 1
    op.mdagm(ap, x)
    for ri, bi, ai in zip(r, b, ap):
        op.axpby(ri, -1.0, ai, bi)
    return k + 1, (op.dot(r, r).real / bb) ** 0.5


# ---- the device-resident form of the decomposed CG ----

class _DeviceOps:
    """the pieces of the decomposed MatPcDagMatPc on one stream, without host
    synchronisation: every slab's lattice launches on `stream`, faces move
    by the ring's enqueued exchange, dot products land in device tensors"""

    def __init__(self, op: DDOperator, stream):
        self.op, self.stream = op, stream
        self.part = torch.zeros((len(op.ops), 2), dtype=torch.float64, device="cuda")

    def dslash(self, out, inp, cb, dag):
        op = self.op
        for D, i, f in zip(op.ops, inp, op.faces):
            pack(D, i, cb, dag, f)
        for D, o, i in zip(op.ops, out, inp):
            dslash_interior(D, o, i, cb, dag)
        op.ring.exchange(op.faces, sync=False)
        for D, o, i, f in zip(op.ops, out, inp, op.faces):
            dslash_boundary(D, o, i, cb, dag, f)

    def matpc(self, out, inp, dag):
        op = self.op
        self.dslash(op.t1, inp, 1, dag)
        self.dslash(out, op.t1, 0, dag)
        for D, o, i in zip(op.ops, out, inp):
            axpby(o, -D.kappa * D.kappa, o, i)

    def dot(self, a, b, out: torch.Tensor) -> None:
        """out[:] = global <a, b> (re, im)"""
        for k, (x, y) in enumerate(zip(a, b)):
            dot_device(x, y, self.part[k])
        torch.sum(self.part, dim=0, out=out)
        self.op.ring.allreduce_device(out)

    def mdagm(self, out, inp, pap: torch.Tensor) -> None:
        self.matpc(self.op.t2, inp, 0)
        self.dot(self.op.t2, self.op.t2, pap)
        self.matpc(out, self.op.t2, 1)


def cg_device(op: DDOperator, x, b, stop_rsd=1e-8, max_num_iter=10000, check_every=8, graph=False):
    """cg's recurrences (InvCgShift, inv_cg.C:84-448) with every scalar on the
    device: alpha, beta and the stop test are device tensors, each global
    sum a device reduction summed over the ranks on the stream (NCCL with
    DistRing), and an iteration after the solve has converged changes
    neither x nor r (alpha = 0; its iteration is not counted), so the host
    looks at the residual only every `check_every` iterations and the
    iteration count is cg's.  graph=True captures one iteration in a CUDA
    graph and replays it.  Returns (iterations + 1, true residual) as cg.
    The solve runs on a stream of its own (ordered after the caller's
    current stream), where the library's launches and torch's scalar
    operations and face copies follow one another."""
    caller = torch.cuda.current_stream()
    stream = torch.cuda.Stream()
    stream.wait_stream(caller)
    with torch.cuda.stream(stream):
        try:
            return _cg_device(op, x, b, stream, stop_rsd, max_num_iter, check_every, graph)
        finally:
            stream.synchronize()
            for D in op.ops:
                set_stream(D.lat, None)
            caller.wait_stream(stream)


def _cg_device(op, x, b, stream, stop_rsd, max_num_iter, check_every, graph):
    """cg_device's body, on `stream` (the current stream)"""
    for D in op.ops:
        set_stream(D.lat, stream)
    dev = _DeviceOps(op, stream)
    r, p, ap = op.field(), op.field(), op.field()
    f64 = dict(dtype=torch.float64, device="cuda")
    bb2, pap2, rr2, rrn2 = (torch.zeros(2, **f64) for _ in range(4))
    alpha, beta, neg_one = torch.zeros(1, **f64), torch.zeros(1, **f64), torch.full((1,), -1.0, **f64)
    iters = torch.zeros(1, **f64)
    dev.dot(b, b, bb2)
    stop = torch.tensor([0.0], **f64)
    torch.mul(bb2[:1], stop_rsd * stop_rsd, out=stop)
    # r = b - A x, p = r, rr = |r|^2
    dev.mdagm(ap, x, pap2)
    for ri, bi, ai in zip(r, b, ap):
        axpby_device(ri, neg_one, 1.0, ai, bi)
    for pi, ri in zip(p, r):
        axpby(pi, 0.0, ri, ri)
    dev.dot(r, r, rr2)

    def step():
        live = (rr2[:1] > stop).to(torch.float64)  # 0 once converged: the step changes nothing
        dev.mdagm(ap, p, pap2)
        torch.where(live > 0, rr2[:1] / pap2[:1], torch.zeros_like(live), out=alpha)
        for xi, pi in zip(x, p):
            axpby_device(xi, alpha, 1.0, pi, xi)
        for ri, ai in zip(r, ap):
            axpby_device(ri, alpha, -1.0, ai, ri)
        dev.dot(r, r, rrn2)
        torch.where(live > 0, rrn2[:1] / rr2[:1], torch.ones_like(live), out=beta)
        rr2.copy_(torch.where(live > 0, rrn2, rr2))
        for pi, ri in zip(p, r):
            axpby_device(pi, beta, 1.0, pi, ri)
        iters.add_(live)

    g = None
    if graph:
        step()  # sizes every buffer before the capture
        side = torch.cuda.Stream()
        side.wait_stream(stream)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            for D in op.ops:
                set_stream(D.lat, side)
            with torch.cuda.graph(g, stream=side):
                step()
        stream.wait_stream(side)
        for D in op.ops:
            set_stream(D.lat, stream)
    k = 1 if graph else 0
    while k < max_num_iter - 1:
        n = min(check_every, max_num_iter - 1 - k)
        for _ in range(n):
            if g is not None:
                g.replay()
            else:
                step()
        k += n
        if float(rr2[0]) <= float(stop[0]):
            break
    done = int(iters.item())
    # true residual (inv_cg.C:403-415)
    dev.mdagm(ap, x, pap2)
    for ri, bi, ai in zip(r, b, ap):
        axpby_device(ri, neg_one, 1.0, ai, bi)
    dev.dot(r, r, rr2)
    true_res = (float(rr2[0]) / float(bb2[0])) ** 0.5
    return done + 1, true_res
