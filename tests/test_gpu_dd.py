"""t-slab domain decomposition of the dslash (the halo exchange that
replaces wilson_dslash_vec's QMP halo, d_op_wilson/qmp/wilson_dslash_vec.C:
184-278).  One process plays every rank: each slab is its own Lattice with
its own links, the faces move between the slabs' device buffers by copies
(what NCCL does between GPUs), and the slabs' outputs together must equal
the whole lattice's dslash and the oracle's."""
import numpy as np
import pytest
import torch

from cps_veloc_b200 import _abi as A
from cps_veloc_b200 import dd
from cps_veloc_b200.dirac import DiracOpDwf, DiracOpWilson, Lattice, gen_gauge, gen_gaussian
from helpers import OracleOps, rel

pytestmark = pytest.mark.gpu


def _slab_gauge(u, L, nodes, r):
    """the links of slab r (WILSON order: [parity][checkerboard site][mu][18], t slowest)"""
    vh = int(np.prod(L)) // 2
    face = vh // L[3]
    lt = L[3] // nodes
    up = u.reshape(2, vh, 72)
    return np.ascontiguousarray(up[:, r * lt * face:(r + 1) * lt * face, :]).ravel()


def _slab_vec(x, L, ls, nodes, r):
    vh = int(np.prod(L)) // 2
    face, lt = vh // L[3], L[3] // nodes
    return np.ascontiguousarray(x.reshape(ls, vh, 24)[:, r * lt * face:(r + 1) * lt * face, :]).ravel()


def _join(parts, L, ls):
    vh = int(np.prod(L)) // 2
    return np.concatenate([p.reshape(ls, -1, 24) for p in parts], axis=1).reshape(ls * vh * 24)


def _make(kind, lat, mass, ls):
    return DiracOpWilson(lat, mass=mass) if kind == "wilson" else DiracOpDwf(lat, mass=mass, ls=ls)


@pytest.mark.parametrize("kind,L,ls,nodes", [("wilson", (4, 4, 4, 8), 1, 2), ("dwf", (4, 4, 4, 8), 4, 2),
                                             ("wilson", (4, 4, 2, 12), 1, 3), ("dwf", (4, 4, 4, 4), 4, 2),
                                             ("wilson", (8, 4, 4, 12), 1, 2)])
@pytest.mark.parametrize("prec", [A.DOUBLE, A.SINGLE])
def test_dd_dslash_matches_whole_lattice(oracle, kind, L, ls, nodes, prec):
    """also: the interior / boundary split (the overlapped form) writes the
    single decomposed launch's output bit for bit, slabs of two t-slices
    (no interior) included"""
    mass = 0.1
    u = gen_gauge(L, seed=501)
    full = Lattice(L)
    full.import_gauge(u)
    Dfull = _make(kind, full, mass, ls)
    lt = L[3] // nodes
    Ls_ = (L[0], L[1], L[2], lt)
    slabs = []
    for r in range(nodes):
        lat = Lattice(Ls_)
        lat.import_gauge(_slab_gauge(u, L, nodes, r))
        dd.set_t_partition(lat, nodes, r)
        D = _make(kind, lat, mass, ls)
        slabs.append((lat, D, dd.DeviceField(D, prec), dd.DeviceField(D, prec), dd.Faces(D, prec),
                      dd.DeviceField(D, prec)))
    ops = OracleOps(oracle, L, u, ls=ls)
    x = gen_gaussian(Dfull.f_size, seed=502)
    for cb in (0, 1):
        for dag in (0, 1):
            for r, (lat, D, fin, fout, fc, fsplit) in enumerate(slabs):
                fin.upload(_slab_vec(x, L, ls, nodes, r))
                dd.pack(D, fin, cb, dag, fc)
                dd.dslash_interior(D, fsplit, fin, cb, dag)
            for r in range(nodes):  # the transport: faces to the neighbouring slabs (periodic)
                slabs[r][4].from_next.copy_(slabs[(r + 1) % nodes][4].to_prev)
                slabs[r][4].from_prev.copy_(slabs[(r - 1) % nodes][4].to_next)
            torch.cuda.synchronize()
            parts = []
            for lat, D, fin, fout, fc, fsplit in slabs:
                dd.dslash(D, fout, fin, cb, dag, fc)
                parts.append(fout.download())
                dd.dslash_boundary(D, fsplit, fin, cb, dag, fc)
                np.testing.assert_array_equal(fsplit.download(), parts[-1])
            y = _join(parts, L, ls)
            whole = Dfull.Dslash(x, cb, dag, prec)
            tol = 1e-14 if prec == A.DOUBLE else 1e-6
            assert rel(y, whole) < tol
            ref = ops.wilson_dslash(x, cb, dag) if kind == "wilson" else ops.dwf_dslash(x, mass, cb, dag)
            assert rel(y, ref) < (1e-13 if prec == A.DOUBLE else 1e-6)


def test_partitioned_lattice_refuses_other_operators():
    L = (4, 4, 4, 4)
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=503))
    dd.set_t_partition(lat, 2, 0)
    D = DiracOpWilson(lat, mass=0.1)
    with pytest.raises(A.CpsGpuError):
        D.MatPc(gen_gaussian(D.f_size, seed=504))
    with pytest.raises(A.CpsGpuError):
        lat.plaquette()
    for nodes_t, coor_t in ((2, 2), (2, -1), (0, 0)):  # coor_t outside [0, nodes_t)
        with pytest.raises(A.CpsGpuError):
            dd.set_t_partition(lat, nodes_t, coor_t)
    with pytest.raises(A.CpsGpuError):  # faces are sized only for FP64 / FP32 fields
        dd.Faces(D, prec=A.HALF)
    dd.set_t_partition(lat, 1, 0)  # back to a whole lattice
    assert D.MatPc(gen_gaussian(D.f_size, seed=504)).size == D.f_size


@pytest.mark.parametrize("kind,L,ls,nodes", [("wilson", (4, 4, 4, 8), 1, 2), ("dwf", (4, 4, 2, 12), 4, 3)])
def test_dd_cg_matches_whole_lattice_solve(kind, L, ls, nodes):
    """CG on MatPcDagMatPc over t slabs (the decomposed MatPc, wilson_m.C /
    dwf_m.C, and InvCgShift's recurrences with every dot product summed over
    the slabs) against the whole lattice's device CG: the same iteration
    count within one, the same solution."""
    mass = 0.1
    u = gen_gauge(L, seed=511)
    full = Lattice(L)
    full.import_gauge(u)
    Dfull = _make(kind, full, mass, ls)
    b = gen_gaussian(Dfull.f_size, seed=512)
    x = np.zeros(Dfull.f_size)
    r = Dfull.InvCg(x, b, stop_rsd=1e-11)
    lt = L[3] // nodes
    ops = []
    for k in range(nodes):
        lat = Lattice((L[0], L[1], L[2], lt))
        lat.import_gauge(_slab_gauge(u, L, nodes, k))
        dd.set_t_partition(lat, nodes, k)
        ops.append((lat, _make(kind, lat, mass, ls)))
    sols = {}
    for overlap in (True, False):
        op = dd.DDOperator([D for _, D in ops], dd.InProcessRing(), overlap=overlap)
        bs, xs = op.field(), op.field()
        for k, (fb, fx) in enumerate(zip(bs, xs)):
            fb.upload(_slab_vec(b, L, ls, nodes, k))
            fx.upload(np.zeros(fx.D.f_size))
        it, tr = dd.cg(op, xs, bs, stop_rsd=1e-11)
        y = _join([f.download() for f in xs], L, ls)
        assert abs(it - r.iterations) <= 1 and tr < 1e-11
        assert rel(y, x) < 1e-9
        sols[overlap] = (it, y)
    # the overlapped operator is the same operator, bit for bit
    assert sols[True][0] == sols[False][0]
    np.testing.assert_array_equal(sols[True][1], sols[False][1])


@pytest.mark.parametrize("kind,L,ls,nodes", [("wilson", (4, 4, 4, 8), 1, 2), ("dwf", (4, 4, 2, 12), 4, 3)])
@pytest.mark.parametrize("graph", [False, True])
def test_dd_device_cg_matches_host_cg(kind, L, ls, nodes, graph):
    """The device-resident decomposed CG (scalars in device tensors, every
    launch enqueued on one stream of its own, the stop test read every 8
    iterations, optionally one iteration captured in a CUDA graph and
    replayed) against
    the host-driven dd.cg on the same slabs: the same iteration count (the
    reductions may round differently: within one) and solution."""
    mass = 0.1
    u = gen_gauge(L, seed=521)
    full = Lattice(L)
    full.import_gauge(u)
    Dfull = _make(kind, full, mass, ls)
    b = gen_gaussian(Dfull.f_size, seed=522)
    lt = L[3] // nodes
    ops = []
    for k in range(nodes):
        lat = Lattice((L[0], L[1], L[2], lt))
        lat.import_gauge(_slab_gauge(u, L, nodes, k))
        dd.set_t_partition(lat, nodes, k)
        ops.append((lat, _make(kind, lat, mass, ls)))
    res = {}
    for device in (False, True):
        op = dd.DDOperator([D for _, D in ops], dd.InProcessRing())
        bs, xs = op.field(), op.field()
        for k, (fb, fx) in enumerate(zip(bs, xs)):
            fb.upload(_slab_vec(b, L, ls, nodes, k))
            fx.upload(np.zeros(fx.D.f_size))
        if device:
            it, tr = dd.cg_device(op, xs, bs, stop_rsd=1e-11, graph=graph)
        else:
            it, tr = dd.cg(op, xs, bs, stop_rsd=1e-11)
        res[device] = (it, tr, _join([f.download() for f in xs], L, ls))
    assert abs(res[True][0] - res[False][0]) <= 1
    assert res[True][1] < 1e-11
    assert rel(res[True][2], res[False][2]) < 1e-9
    # the legacy default stream (a null handle) cannot be named as a lattice's stream
    with pytest.raises(ValueError):
        dd.set_stream(ops[0][0], torch.cuda.default_stream())
