"""Host logic of the product library on CPU: exported C ABI, quadrature, and the sweep schedule
(bit-exact against the oracle's literal restatement of SweepOrder.f90 / SweepArrays.f90).
These tests use host-only handles (lb_create(-1)): no GPU, no kernel launches."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O
from helpers import golden, golden_mesh, jittered
from lionbolt_b200 import _lib
from lionbolt_b200 import mesh as M
from lionbolt_b200 import problems as P

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "lionbolt_b200.h")


def header_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(lb_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
        assert s in _lib.SIGNATURES, f"{s} missing from the ctypes signature table"


def _givens(x, y):
    lib = _lib.load()
    c, s, r = np.zeros(1), np.zeros(1), np.zeros(1)
    assert lib.lb_givens(x, y, _lib.dptr(c), _lib.dptr(s), _lib.dptr(r)) == 0
    return c[0], s[0], r[0]


def test_givens_rotation_follows_sparskit():
    """iters.f:3225-3262: (x, y) -> (r, 0), including its branch for NaN input (identity, r = 0)."""
    for x, y in [(3.0, 4.0), (-4.0, 3.0), (1e-300, -2.0), (5.0, 0.0)]:
        c, s, r = _givens(x, y)
        assert abs(c * x + s * y - r) <= 1e-15 * max(1.0, r) and abs(-s * x + c * y) <= 1e-15 * max(1.0, r)
        assert abs(r - np.hypot(x, y)) <= 1e-15 * r and abs(c * c + s * s - 1.0) < 1e-15
    assert _givens(0.0, 0.0) == (1.0, 0.0, 0.0)
    for x, y in [(np.nan, 1.0), (1.0, np.nan), (np.nan, np.nan)]:
        assert _givens(x, y) == (1.0, 0.0, 0.0)


def test_status_strings():
    lib = _lib.load()
    assert lib.lb_status_string(0) == b"ok"
    assert b"stagnant" in lib.lb_status_string(_lib.LB_ERR_CYCLE)


@pytest.mark.parametrize("L,fname", [(11, "ordinates_L11.txt"), (7, "ordinates_L7.txt")])
def test_product_quadrature_matches_reference_log(L, fname):
    k, w = _lib.sn_quadrature(L + 1, 2 * (L + 1))
    assert np.abs(k - golden(fname)).max() < 2.5e-16
    assert abs(w.sum() - 4 * np.pi) < 1e-13


class HostHandle:
    def __init__(self):
        self.lib = _lib.load()
        self.h = ctypes.c_void_p()
        assert self.lib.lb_create(-1, ctypes.byref(self.h)) == 0

    def mesh(self, m):
        return self.lib.lb_set_mesh(self.h, m.NE, m.NN, _lib.dptr(_lib.as_f64(m.rg)), _lib.iptr(_lib.as_i32(m.node)),
                                    _lib.iptr(_lib.as_i32(m.neighbors)), _lib.iptr(_lib.as_i32(m.mat)), int(m.Nm))

    def quad(self, k, w):
        return self.lib.lb_set_quadrature(self.h, k.shape[0], _lib.dptr(_lib.as_f64(k)), _lib.dptr(_lib.as_f64(w)))

    def schedule(self, NE, NI):
        sl = np.zeros((NI, NE), np.int32)
        up = np.zeros((NI, NE), np.uint8)
        nl = np.zeros(NI, np.int32)
        ls = np.zeros((NI, NE + 1), np.int32)
        assert self.lib.lb_get_schedule(self.h, _lib.iptr(sl), up.ctypes.data_as(_lib._c_ubyte_p), _lib.iptr(nl),
                                        _lib.iptr(ls)) == 0
        return sl, up, nl, ls

    def error(self):
        buf = ctypes.create_string_buffer(256)
        self.lib.lb_last_error(self.h, buf, 256)
        return buf.value.decode()

    def __del__(self):
        self.lib.lb_destroy(self.h)


def reference_arrays_from_product(sl, up, m):
    """Derive SweepArrays.f90 arrays (UFoffset, upfaces, ipsf) from the product's schedule."""
    NI, NE = sl.shape
    isl = np.empty_like(sl)
    for i in range(NI):
        isl[i, sl[i]] = np.arange(NE)
    upf, ipsf, UF = [], [], np.zeros((NI, NE + 1), np.int64)
    j = 0
    for i in range(NI):
        for es in range(NE):
            e = sl[i, es]
            UF[i, es] = j
            for f in range(4):
                if (up[i, es] >> f) & 1:
                    upf.append(f)
                    ep = m.neighbors[e, f]
                    ipsf.append(i * 4 * NE + 4 * isl[i, ep])
                    j += 1
        UF[i, NE] = j
    return isl, np.array(upf, np.int32), np.array(ipsf, np.int64), UF


CASES = {
    "config0": lambda: (P.config0().mesh, P.quadrature(8, 10)),
    "two_material": lambda: (P.config1_small(n=(4, 4, 8)).mesh, P.quadrature(6, 12)),
    "jittered": lambda: (jittered(M.box_mesh(5, 4, 3, (0, 0, 0), (2.5, 2.0, 1.5)), 0.06), P.quadrature(4, 8)),
    "L11_288": lambda: (M.box_mesh(3, 3, 6, (0, 0, 0), (1.5, 1.5, 3.0)), P.quadrature(12, 24)),
    # unstructured gmsh meshes of the reference (tests/golden fixtures of its shipped .msh files)
    "gmsh_simple_cube": lambda: (golden_mesh("simple_cube"), P.quadrature(4, 8)),
    "gmsh_het_cube": lambda: (golden_mesh("het_cube_spherical_beam"), P.quadrature(2, 4)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_schedule_bitexact_vs_literal_sweep_order(case):
    m, (k, w) = CASES[case]()
    o = O.Oracle(m)
    assert o.set_angular(k, w, 0, literal=True) == 0
    ref = o.schedule()
    hh = HostHandle()
    assert hh.mesh(m) == 0, hh.error()
    assert hh.quad(k, w) == 0, hh.error()
    sl, up, nl, ls = hh.schedule(m.NE, k.shape[0])
    assert np.array_equal(sl, ref["sl"])
    assert np.array_equal(nl, ref["nlevels"])
    isl, upf, ipsf, UF = reference_arrays_from_product(sl, up, m)
    assert np.array_equal(isl, ref["isl"])
    assert np.array_equal(upf, ref["upfaces"])
    assert np.array_equal(ipsf, ref["ipsf"])
    assert np.array_equal(UF, ref["UFoffset"])
    # level starts: contiguous, ascending element ids inside every level
    for i in range(0, k.shape[0], max(1, k.shape[0] // 7)):
        st = ls[i, :nl[i] + 1]
        assert st[0] == 0 and st[-1] == m.NE
        for a, b in zip(st[:-1], st[1:]):
            assert np.all(np.diff(sl[i, a:b]) > 0)


def test_empty_and_invalid_meshes_are_rejected():
    hh = HostHandle()
    lib = hh.lib
    z = np.zeros(12)
    zi = np.zeros(4, np.int32)
    assert lib.lb_set_mesh(hh.h, 0, 4, _lib.dptr(z), _lib.iptr(zi), _lib.iptr(zi), _lib.iptr(zi), 1) == _lib.LB_ERR_ARG
    m = M.box_mesh(1, 1, 1)
    bad = m.node.copy()
    bad[0, 0] = m.NN + 5
    assert lib.lb_set_mesh(hh.h, m.NE, m.NN, _lib.dptr(_lib.as_f64(m.rg)), _lib.iptr(_lib.as_i32(bad)),
                           _lib.iptr(_lib.as_i32(m.neighbors)), _lib.iptr(_lib.as_i32(m.mat)), 1) == _lib.LB_ERR_ARG
    # quadrature before a mesh: operator not ready
    hh2 = HostHandle()
    k, w = P.quadrature(2, 4)
    assert hh2.quad(k, w) == _lib.LB_ERR_STATE
    # non-conforming neighbour table
    nb = m.neighbors.copy()
    nb[0, :] = -1
    m2 = M.Mesh(rg=m.rg, node=m.node, neighbors=nb, mat=m.mat, Nm=1)
    assert hh.mesh(m2) == _lib.LB_ERR_ARG


def test_folded_mesh_cycle_is_reported():
    """Two tets on the same side of their shared face both see it as an inflow face for some
    direction: the level loop stagnates, which the reference reports as 'Sweep is stagnant'."""
    rg = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.2, 0.2, 1.0], [0.3, 0.25, 0.5]], dtype=np.float64)
    node = np.array([[0, 1, 2, 3], [0, 2, 1, 4]], dtype=np.int32)   # both apexes above the z=0 face
    nb = np.array([[1, -1, -1, -1], [1 * 0, -1, -1, -1]], dtype=np.int32)
    nb[1, 0] = 0
    m = M.Mesh(rg=rg, node=node, neighbors=nb, mat=np.zeros(2, np.int32), Nm=1)
    hh = HostHandle()
    assert hh.mesh(m) == 0, hh.error()
    k = np.array([[0.0, 0.0, 1.0]])
    w = np.array([4 * np.pi])
    assert hh.quad(k, w) == _lib.LB_ERR_CYCLE
    assert "stagnant" in hh.error()


def test_host_only_handle_refuses_compute():
    m = M.box_mesh(1, 1, 1)
    hh = HostHandle()
    assert hh.mesh(m) == 0
    k, w = P.quadrature(2, 4)
    assert hh.quad(k, w) == 0
    s = np.zeros(m.NENK * k.shape[0])
    assert hh.lib.lb_transport_inv(hh.h, _lib.dptr(s)) == _lib.LB_ERR_STATE


def test_nan_cross_section_rejected():
    m = M.box_mesh(1, 1, 1)
    hh = HostHandle()
    hh.mesh(m)
    k, w = P.quadrature(2, 4)
    hh.quad(k, w)
    st = np.array([np.nan])
    ss = np.zeros((1, 2))
    assert hh.lib.lb_set_xs(hh.h, 1, _lib.dptr(st), _lib.dptr(ss)) == _lib.LB_ERR_NAN


def test_element_type_table():
    """Box meshes have 6 element shapes (the Kuhn split) per material, so the sweep reads 16-byte
    records and a per-type table; a jittered mesh has a shape per element and keeps 64-byte records."""
    n = np.zeros(1, np.int32)
    hh = HostHandle()
    assert hh.lib.lb_mesh_types(hh.h, _lib.iptr(n)) == _lib.LB_ERR_STATE
    assert hh.mesh(M.box_mesh(4, 4, 4)) == 0
    assert hh.lib.lb_mesh_types(hh.h, _lib.iptr(n)) == 0 and n[0] == 6
    two = M.box_mesh(4, 4, 8, (0, 0, 0), (2, 2, 4), material=lambda c: (c[:, 2] > 2.0).astype(np.int32), Nm=2)
    assert hh.mesh(two) == 0
    assert hh.lib.lb_mesh_types(hh.h, _lib.iptr(n)) == 0 and n[0] == 12
    jit = jittered(M.box_mesh(6, 5, 4, (0, 0, 0), (3.0, 2.5, 2.0)), 0.07)
    assert jit.NE > 256
    assert hh.mesh(jit) == 0
    assert hh.lib.lb_mesh_types(hh.h, _lib.iptr(n)) == 0 and n[0] == 0


def _cluster_schedule(hh, NE, NI):
    nb, ml = np.zeros(1, np.int32), np.zeros(1, np.int32)
    assert hh.lib.lb_cluster_info(hh.h, _lib.iptr(nb), _lib.iptr(ml)) == 0
    if nb[0] == 0:
        return None
    base = np.zeros(NI + 1, np.int64)
    mem = np.zeros((nb[0], 6), np.int32)
    mr = np.zeros(1, np.int32)
    assert hh.lib.lb_cluster_layout(hh.h, base.ctypes.data_as(_lib._c_ll_p), _lib.iptr(mem), _lib.iptr(mr)) == 0
    rec = np.zeros((base[NI], 4), np.int32)
    st = np.zeros((NI, mr[0] + 1), np.int32)
    nl = np.zeros(NI, np.int32)
    assert hh.lib.lb_get_cluster_schedule(hh.h, _lib.iptr(rec), _lib.iptr(st), _lib.iptr(nl)) == 0
    return dict(nb=int(nb[0]), max_levels=int(ml[0]), base=base, members=mem, rec=rec, starts=st, nlevels=nl)


def _check_cluster_schedule(m, k, w):
    """Every element once per direction with the reference's upstream mask, every record's elements
    members of its block, every upstream neighbour in another record on an earlier block level and
    every upstream neighbour in the same record in an earlier slot."""
    hh = HostHandle()
    assert hh.mesh(m) == 0 and hh.quad(k, w) == 0, hh.error()
    NE, NI = m.NE, k.shape[0]
    sl, up, nlev, ls = hh.schedule(NE, NI)
    cs = _cluster_schedule(hh, NE, NI)
    assert cs is not None
    mem = cs["members"]
    assert sorted(mem[mem >= 0].tolist()) == list(range(NE))
    nbr = m.neighbors
    split = 0
    far = 0
    for i in range(NI):
        upm = np.zeros(NE, np.int64)
        upm[sl[i]] = up[i]
        rec = cs["rec"][cs["base"][i]:cs["base"][i + 1]]
        nr = rec.shape[0]
        split += nr - cs["nb"]
        rec_level = np.empty(nr, np.int64)
        st = cs["starts"][i]
        for L in range(cs["nlevels"][i]):
            rec_level[st[L]:st[L + 1]] = L
        assert st[cs["nlevels"][i]] == nr
        words = rec[:, 1:].astype(np.uint32)
        slots = np.stack([words & 0xFFFF, words >> 16], axis=2).reshape(nr, 6)
        off = slots & 7
        seen = np.zeros(NE, np.int64)
        rec_of = np.full(NE, -1, np.int64)
        slot_of = np.full(NE, -1, np.int64)
        for r in range(nr):
            for kk in range(6):
                if off[r, kk] == 7:
                    continue
                e = int(mem[rec[r, 0], off[r, kk]])
                assert e >= 0
                seen[e] += 1
                rec_of[e], slot_of[e] = r, kk
                assert ((slots[r, kk] >> 3) & 15) == upm[e]
        assert np.all(seen == 1)
        for f in range(4):
            e = np.nonzero((upm >> f) & 1)[0]
            ne = nbr[e, f]
            other = rec_of[ne] != rec_of[e]
            assert np.all(rec_level[rec_of[ne[other]]] < rec_level[rec_of[e[other]]])
            assert np.all(slot_of[ne[~other]] < slot_of[e[~other]])
            # walk distance of every in-block upstream read (the kernels hold the last two solutions)
            far += int(np.count_nonzero(slot_of[e[~other]] - slot_of[ne[~other]] > 2))
    cs["far_reads"] = far
    return cs, split


def test_cluster_schedule_respects_every_dependency():
    """The block schedule against the reference schedule.  A box mesh: blocks of 6 consecutive tets
    (one hex), nx + ny + nz - 2 block levels in an oblique direction, no block split, and walk orders
    that read every in-block upstream neighbour within two updates.  A jittered
    box: blocks on dependency cycles are split into single elements in the directions that need it.
    The reference's unstructured meshes: blocks grown from face neighbours."""
    m = P.config1_small(n=(6, 6, 12)).mesh
    hh = HostHandle()
    nb0, ml0 = np.zeros(1, np.int32), np.zeros(1, np.int32)
    assert hh.lib.lb_cluster_info(hh.h, _lib.iptr(nb0), _lib.iptr(ml0)) == _lib.LB_ERR_STATE   # no quadrature yet
    cs, split = _check_cluster_schedule(m, *P.quadrature(6, 12))
    assert cs["nb"] == m.NE // 6 and cs["max_levels"] == 6 + 6 + 12 - 2 and split == 0
    assert np.array_equal(cs["members"].ravel(), np.arange(m.NE))
    # each block's walk order leaves every in-block upstream neighbour among the two previous updates
    assert cs["far_reads"] == 0
    jit = jittered(M.box_mesh(6, 5, 4, (0, 0, 0), (3.0, 2.5, 2.0)), 0.07)
    cs, split = _check_cluster_schedule(jit, *P.quadrature(4, 8))
    assert split > 0
    for name, quad in (("simple_cube", (4, 8)), ("het_cube_spherical_beam", (2, 4))):
        g = golden_mesh(name)
        cs, split = _check_cluster_schedule(g, *P.quadrature(*quad))
        sizes = (cs["members"] >= 0).sum(axis=1)
        assert sizes.mean() > 4.5, (name, sizes.mean())        # mostly full blocks
        assert split > 0                                        # block graphs of unstructured meshes have cycles


def test_cluster_groups_are_capped_and_packed(monkeypatch):
    """Groups of the block schedule hold at most one unit per sweep thread (the cap, here 16 instead of
    512): a level with more ready units spills into the next group, which the units that became ready
    meanwhile fill up, so the groups take fewer passes of the CTA than Kahn's levels do, and every
    dependency still points to an earlier group (checked by _check_cluster_schedule)."""
    m = M.box_mesh(8, 8, 8, (0, 0, 0), (1, 1, 1))
    k, w = P.quadrature(4, 8)
    monkeypatch.setenv("LB_CLUSTER_GROUP", "0")
    levels, _ = _check_cluster_schedule(m, k, w)
    monkeypatch.setenv("LB_CLUSTER_GROUP", "16")
    groups, split = _check_cluster_schedule(m, k, w)
    assert split == 0
    passes_levels = passes_groups = 0
    for i in range(k.shape[0]):
        nl = np.diff(levels["starts"][i][: levels["nlevels"][i] + 1])
        ng = np.diff(groups["starts"][i][: groups["nlevels"][i] + 1])
        assert ng.max() <= 16 and nl.max() > 16
        passes_levels += int(np.sum((nl + 15) // 16))
        passes_groups += len(ng)
    assert passes_groups < passes_levels


def test_pipeline_timeout_probe_needs_a_device_and_a_bound():
    hh = HostHandle()
    assert hh.lib.lb_probe_pipeline_timeout(hh.h, 0) == _lib.LB_ERR_ARG
    assert hh.lib.lb_probe_pipeline_timeout(hh.h, 4096) == _lib.LB_ERR_STATE   # host-only handle


def test_cluster_queries_need_a_block_schedule():
    hj = HostHandle()
    assert hj.mesh(M.box_mesh(1, 1, 1)) == 0 and hj.quad(*P.quadrature(2, 4)) == 0
    nb, ml = np.zeros(1, np.int32), np.zeros(1, np.int32)
    assert hj.lib.lb_cluster_info(hj.h, _lib.iptr(nb), _lib.iptr(ml)) == 0 and nb[0] == 1
    hs = HostHandle()
    assert hs.mesh(M.box_mesh(1, 1, 1)) == 0
    one = np.zeros(4, np.int32)
    assert hs.lib.lb_get_cluster_schedule(hs.h, _lib.iptr(one), _lib.iptr(one), _lib.iptr(one)) == _lib.LB_ERR_STATE
