"""The results-file writer (lionbolt_b200/lionbolt_hdf5.py: the reference's LionboltHDF5.f90 without
the HDF5 library).  CPU only.

Pins: (1) the reader reads a file that the HDF5 library wrote (scipy's MATLAB 7.4 test file, a
classic-format HDF5 file with a 512-byte user block); (2) the writer encodes the same object (a
[9, 1] float64 dataset with a string attribute) in exactly the library's bytes, the data address
aside; (3) every member of every group is found by the library's B-tree descent (key_i < name <=
key_{i+1}, then binary search in the symbol-table node), including groups large enough for a
two-level B-tree; (4) the Lionbolt layout of schema.yaml round-trips."""
import os
import struct

import numpy as np
import pytest
import scipy

from lionbolt_b200 import lionbolt_hdf5 as H
from lionbolt_b200 import mesh as M
from lionbolt_b200 import problems as P

LIB_FILE = os.path.join(os.path.dirname(scipy.__file__), "io", "matlab", "tests", "data", "testhdf5_7.4_GLNX86.mat")
needs_lib_file = pytest.mark.skipif(not os.path.exists(LIB_FILE), reason="scipy's HDF5 test file is not installed")


def _dataset_messages(path, name):
    """{message type: (flags, data bytes)} of a dataset in the root group."""
    r = H._Reader(path)
    for t, p, _ in r.messages(r.root_oh):
        if t == H.MSG_STAB:
            btree, heap = struct.unpack_from("<QQ", r.b, p)
    oh = _lookup(r, btree, heap, name)
    return {t: (r.b[p - 4], r.b[p:p + s]) for t, p, s in r.messages(oh)}


def _name(r, heap, off):
    daddr = r.u("<4sB3xQQQ", heap)[4]
    s = r.base + daddr + off
    return r.b[s:r.b.index(b"\0", s)]


def _lookup(r, btree, heap, name):
    """The HDF5 library's lookup of a group member: descend the B-tree choosing the child i with
    key_i < name <= key_{i+1}, then binary-search the symbol-table node's sorted entries."""
    name = name.encode() if isinstance(name, str) else name
    addr = btree
    while True:
        sig, typ, lev, n = r.u("<4sBBH", addr)
        assert sig == b"TREE" and typ == 0
        keys = [_name(r, heap, r.u("<Q", addr + 24 + 16 * i)[0]) for i in range(n + 1)]
        kids = [r.u("<Q", addr + 32 + 16 * i)[0] for i in range(n)]
        assert keys == sorted(keys) and len(set(keys)) == len(keys)
        lo, hi = 0, n
        while lo < hi:                       # binary search over the children
            mid = (lo + hi) // 2
            if name <= keys[mid]:
                hi = mid
            elif name > keys[mid + 1]:
                lo = mid + 1
            else:
                lo = hi = mid
        assert lo < n and keys[lo] < name <= keys[lo + 1], name
        if lev == 0:
            break
        addr = kids[lo]
    snod = kids[lo]
    sig, _, _, ns = r.u("<4sBBH", snod)
    assert sig == b"SNOD"
    ents = [r.u("<QQ", snod + 8 + 40 * j) for j in range(ns)]
    names = [_name(r, heap, e[0]) for e in ents]
    assert names == sorted(names)
    assert names[-1] == keys[lo + 1]          # the right key is the node's largest name
    j = int(np.searchsorted(np.array(names, dtype=object), name))
    assert names[j] == name
    return ents[j][1]


def _check_group_lookups(path):
    """Every member of every group is found by the library's lookup."""
    r = H._Reader(path)

    def visit(oh):
        for t, p, _ in r.messages(oh):
            if t == H.MSG_STAB:
                btree, heap = struct.unpack_from("<QQ", r.b, p)
                members = r.group(btree, heap)
                for nm in members:
                    child = _lookup(r, btree, heap, nm)
                    visit(child)
                return len(members)
        return 0

    return visit(r.root_oh)


@needs_lib_file
def test_reader_reads_a_file_written_by_the_hdf5_library():
    f = H.read(LIB_FILE)
    assert list(f) == ["testdouble"]
    d = f["testdouble"]
    assert d.shape == (9, 1) and d.dtype == np.float64
    assert np.array_equal(d.ravel(), np.arange(9) * np.pi / 4)
    assert d.attrs == {"MATLAB_class": "double"}
    assert _check_group_lookups(LIB_FILE) == 1


@needs_lib_file
def test_writer_encodes_a_dataset_as_the_hdf5_library_does(tmp_path):
    out = str(tmp_path / "t.h5")
    with H.H5Writer(out) as w:
        d = w.create_dataset("testdouble", (np.arange(9) * np.pi / 4).reshape(9, 1))
        d.attrs["MATLAB_class"] = b"double"
    lib, ours = _dataset_messages(LIB_FILE, "testdouble"), _dataset_messages(out, "testdouble")
    # the library adds a modification time (optional) and pads the header with a NIL message
    assert set(ours) == {H.MSG_FILL, H.MSG_DATATYPE, H.MSG_DATASPACE, H.MSG_LAYOUT, H.MSG_ATTRIBUTE}
    for t in ours:
        if t == H.MSG_LAYOUT:     # version, rank + 1, class, reserved | address | dims, element size
            assert lib[t][0] == ours[t][0]
            assert lib[t][1][:8] == ours[t][1][:8] and lib[t][1][16:] == ours[t][1][16:]
        else:
            assert lib[t] == ours[t], t
    assert np.array_equal(H.read(out)["testdouble"], H.read(LIB_FILE)["testdouble"])


def test_groups_attributes_and_types_round_trip(tmp_path):
    out = str(tmp_path / "g.h5")
    rng = np.random.default_rng(0)
    big = {f"angle_{i + 1}": rng.normal(size=5) for i in range(700)}     # > 256 members: a two-level B-tree
    with H.H5Writer(out) as w:
        w.set_attr("", "problem_type", "general")
        w.create_group("empty")
        w.create_group("a/b/c")
        w.set_attr("a/b", "n", np.int32(7))
        w.set_attr("a/b", "x", 2.5)
        w.create_dataset("a/b/c/i32", np.arange(-3, 9, dtype=np.int32).reshape(3, 4))
        w.create_dataset("a/b/c/i64", np.arange(5, dtype=np.int64))         # stored as Fortran integers
        w.create_dataset("a/b/c/u8", np.arange(5, dtype=np.uint8))
        w.create_dataset("a/b/c/f32", np.linspace(0, 1, 7, dtype=np.float32))
        w.create_dataset("a/b/c/none", np.zeros(0))
        for k, v in big.items():
            w.create_dataset(f"big/{k}", v)
    f = H.read(out)
    assert f.attrs == {"problem_type": "general"}
    assert sorted(f) == ["a", "big", "empty"] and len(f["empty"]) == 0
    assert f["a"]["b"].attrs == {"n": 7, "x": 2.5}
    c = f["a"]["b"]["c"]
    assert c["i32"].dtype == np.int32 and np.array_equal(c["i32"], np.arange(-3, 9).reshape(3, 4))
    assert c["i64"].dtype == np.int32 and np.array_equal(c["i64"], np.arange(5))
    assert c["u8"].dtype == np.uint8 and np.array_equal(c["u8"], np.arange(5))
    assert c["f32"].dtype == np.float32 and np.array_equal(c["f32"], np.linspace(0, 1, 7, dtype=np.float32))
    assert c["none"].shape == (0,)
    assert len(f["big"]) == 700 and all(np.array_equal(f["big"][k], v) for k, v in big.items())
    assert _check_group_lookups(out) == 3
    # the file ends where the superblock says
    eof = struct.unpack_from("<Q", open(out, "rb").read(48), 40)[0]
    assert eof == os.path.getsize(out)


def test_results_file_has_the_reference_layout(tmp_path):
    prob = P.multigroup_box(n=(3, 2, 4), size=(3.0, 2.0, 4.0), G=3, Ng=2, Nc=4, slab=(1.0, 2.0))
    m = prob.mesh
    G, NENK = prob.G, m.NENK
    rng = np.random.default_rng(1)
    flux, dose = rng.uniform(size=(G, NENK)), rng.uniform(size=NENK)
    unc = np.zeros_like(flux)
    unc[0] = prob.unc
    out = H.write_results(str(tmp_path / "lb.h5"), m, prob.w, prob.k, flux, dose, particle="Photon",
                          energy_grid=prob.energy, uncollided=unc)
    f = H.read(out)
    assert f.attrs == {"problem_type": "general"}
    assert sorted(f) == ["dose_deposition", "mesh", "photon"]
    mesh = f["mesh"]
    assert mesh.attrs == {"problem_type": "general", "number_of_materials": 2, "number_of_elements": m.NE,
                          "number_of_spatial_dofs": NENK, "number_of_global_nodes": m.NN}
    # one-based connectivity(offset(e) + k) = global node of (e, k)
    c, o = mesh["connectivity"], mesh["offset"]
    assert c.dtype == np.int32 and o.dtype == np.int32 and o.shape == (m.NE + 1,) and o[-1] == NENK
    e = np.arange(m.NE)
    for k in range(4):
        assert np.array_equal(c[o[:-1] + k] - 1, m.node[e, k])
    assert np.array_equal(mesh["global_nodes"], m.rg)
    assert np.isclose(mesh["element_volumes"].sum(), 3.0 * 2.0 * 4.0)
    sd = mesh["material_to_spatial_dof"]
    assert sorted(sd) == ["material_1", "material_2"]
    both = np.sort(np.concatenate([sd["material_1"], sd["material_2"]]))
    assert np.array_equal(both, np.arange(1, NENK + 1))
    assert np.all(np.repeat(m.mat, 4)[sd["material_2"] - 1] == 1)
    ph = f["photon"]
    assert ph.attrs == {"object_type": "particle", "number_of_energy_dofs": G, "number_of_angular_dofs": prob.NI}
    assert np.array_equal(ph["energy_grid"], prob.energy)
    assert np.array_equal(ph["angular_weights"], prob.w) and np.array_equal(ph["abscissae"], prob.k)
    assert sorted(ph["fluence"]) == [f"energy_{g + 1}" for g in range(G)]
    for g in range(G):
        assert np.array_equal(ph["fluence"][f"energy_{g + 1}"], flux[g])
    assert list(ph["uncollided_fluence"]) == ["energy_1"]
    assert np.array_equal(ph["uncollided_fluence"]["energy_1"], prob.unc)
    assert np.array_equal(f["dose_deposition"], dose)
    _check_group_lookups(out)


def test_angular_fluence_groups(tmp_path):
    m = M.box_mesh(2, 2, 2, (0, 0, 0), (1.0, 1.0, 1.0))
    k, w = P.quadrature(12, 24)                      # 288 angles: a two-level B-tree per group
    NI, NENK = w.size, m.NENK
    x = np.random.default_rng(2).normal(size=NI * NENK)
    with H.ResultsFile(str(tmp_path / "a.h5")) as out:
        out.open_particle("electron")
        out.append_ordinates(w, k)
        out.append_angular_fluence(x, NENK, False, 1)
        out.append_angular_fluence(2 * x, NENK, True, 1)
        out.close_particle("electron")
    f = H.read(str(tmp_path / "a.h5"))
    af, au = f["electron"]["angular_fluence"]["energy_1"], f["electron"]["uncollided_angular_fluence"]["energy_1"]
    assert len(af) == NI == 288
    for i in range(NI):
        assert np.array_equal(af[f"angle_{i + 1}"], x[i * NENK:(i + 1) * NENK])
        assert np.array_equal(au[f"angle_{i + 1}"], 2 * x[i * NENK:(i + 1) * NENK])
    # the fluence of the angular fluence (LinearOperatorClass.f90:154-174)
    fl = sum(w[i] * af[f"angle_{i + 1}"] for i in range(NI))
    assert np.allclose(fl, (w[:, None] * x.reshape(NI, NENK)).sum(axis=0))
    _check_group_lookups(str(tmp_path / "a.h5"))


def test_particle_group_is_tagged_once_and_reopened(tmp_path):
    with H.ResultsFile(str(tmp_path / "p.h5")) as out:
        out.open_particle("Electron")
        out.append_spatial_array("fluence", np.ones(4), 1)
        out.close_particle()
        out.open_particle("ELECTRON")                   # lower-cased: the same group
        out.append_spatial_array("fluence", np.zeros(4), 2)
        out.open_particle("Electron", nolc=True)        # kept as given: another group
        out.close_particle()
    f = H.read(str(tmp_path / "p.h5"))
    assert sorted(f) == ["Electron", "electron"]
    assert f["electron"].attrs == {"object_type": "particle"}
    assert sorted(f["electron"]["fluence"]) == ["energy_1", "energy_2"]
    with pytest.raises(ValueError):
        with H.H5Writer(str(tmp_path / "q.h5")) as w:
            w.create_dataset("d", np.ones(2))
            w.create_dataset("d", np.ones(2))
