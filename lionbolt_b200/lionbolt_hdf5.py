"""Lionbolt results files (src/IO/LionboltHDF5.f90:15-344, names from src/IO/schema.yaml), written in
the HDF5 file format without the HDF5 library.

The files use HDF5's original structures, which every HDF5 reader accepts:
  * a version-0 superblock (offsets and lengths of 8 bytes, group leaf K = 4, internal K = 16,
    the library's defaults);
  * version-1 object headers;
  * groups stored as symbol tables: a version-1 B-tree (type 0) over symbol-table nodes ("SNOD"),
    with the member names in a local heap ("HEAP");
  * contiguous, little-endian datasets in C order (a Fortran array a(3, NK) is the dataset
    [NK, 3], as the Fortran HDF5 interface stores it), attributes as version-1 attribute messages.
Every structure is encoded as the HDF5 library (1.6/1.8) writes it for the same object; the tests
compare the encodings with a file the library wrote.

Raw data go to the file as datasets are added (the angular fluence of a group never has to be held
whole); the metadata follow at close, and the superblock at offset 0 is written last.

`read` is a small reader of the same structures (plus the version-2/3 dataspace, datatype and
layout messages of later library versions), for checking and for users without h5py.
"""
import struct

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
LEAF_K = 4                    # a symbol-table node holds up to 2 * LEAF_K members
NODE_K = 16                   # a B-tree node has up to 2 * NODE_K children
SNOD_SIZE = 8 + 2 * LEAF_K * 40
TREE_SIZE = 24 + 2 * NODE_K * 8 + (2 * NODE_K + 1) * 8
SUPERBLOCK_SIZE = 96

# message types
MSG_NIL, MSG_DATASPACE, MSG_DATATYPE, MSG_FILL, MSG_LAYOUT, MSG_ATTRIBUTE, MSG_STAB = 0, 1, 3, 5, 8, 12, 17


def _pad8(b):
    return b + b"\0" * (-len(b) % 8)


def _datatype(dt):
    """Datatype message, version 1 (unpadded)."""
    dt = np.dtype(dt)
    if dt.kind == "f" and dt.itemsize in (4, 8):
        # class 1; byte order LE, implied mantissa MSB (normalisation 2), sign bit location
        if dt.itemsize == 8:
            return struct.pack("<4BI", 0x11, 0x20, 63, 0, 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        return struct.pack("<4BI", 0x11, 0x20, 31, 0, 4) + struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
    if dt.kind in "iu" and dt.itemsize in (1, 2, 4, 8):
        # class 0; byte order LE, bit 3 = signed
        return struct.pack("<4BI", 0x10, 0x08 if dt.kind == "i" else 0x00, 0, 0, dt.itemsize) + \
            struct.pack("<HH", 0, 8 * dt.itemsize)
    if dt.kind == "S":
        # class 3; null-terminated ASCII
        return struct.pack("<4BI", 0x13, 0x00, 0, 0, dt.itemsize)
    raise TypeError(f"no HDF5 encoding for dtype {dt}")


def _dataspace(shape):
    """Dataspace message, version 1 (rank 0 = scalar)."""
    return struct.pack("<4BI", 1, len(shape), 0, 0, 0) + b"".join(struct.pack("<Q", int(d)) for d in shape)


def _fill():
    """Fill-value message, version 1: allocation late, write if set, default value."""
    return struct.pack("<4BI", 1, 2, 2, 1, 0)


def _layout(shape, itemsize, addr):
    """Data-layout message, version 2, contiguous: dimensions in 4-byte fields, element size last."""
    dims = list(shape) + [itemsize]
    if any(d > 0xFFFFFFFF for d in dims):
        raise ValueError("a dimension exceeds 2^32 - 1 elements")
    return struct.pack("<3B5xQ", 2, len(dims), 1, addr) + b"".join(struct.pack("<I", int(d)) for d in dims)


def _attribute(name, value):
    """Attribute message, version 1: name, datatype and dataspace each padded to 8 bytes."""
    if isinstance(value, str):
        value = value.encode("ascii")
    if isinstance(value, bytes):
        arr = np.array(value, dtype=f"S{max(1, len(value))}")
    else:
        arr = np.asarray(value)
        if arr.dtype.kind == "i" and arr.dtype.itemsize != 4 and np.all(np.abs(arr) < 2**31):
            arr = arr.astype(np.int32)            # Fortran default integer
        arr = np.ascontiguousarray(arr, dtype=arr.dtype.newbyteorder("<"))
    nb = name.encode("ascii") + b"\0"
    dt, ds = _datatype(arr.dtype), _dataspace(arr.shape)
    return struct.pack("<BBHHH", 1, 0, len(nb), len(dt), len(ds)) + _pad8(nb) + _pad8(dt) + _pad8(ds) + arr.tobytes()


def _object_header(msgs):
    """Version-1 object header: 16-byte prefix, then (type, size, flags) messages padded to 8 bytes; a
    NIL message fills the message area up to 32 bytes, as the library allocates it."""
    body = b"".join(struct.pack("<HHB3x", t, len(_pad8(d)), f) + _pad8(d) for t, f, d in msgs)
    n = len(msgs)
    if len(body) < 32:
        body += struct.pack("<HHB3x", MSG_NIL, 32 - len(body) - 8, 0) + b"\0" * (32 - len(body) - 8)
        n += 1
    return struct.pack("<BBHII4x", 1, 0, n, 1, len(body)) + body


class _Group:
    def __init__(self):
        self.members = {}      # name -> _Group | _Dataset
        self.attrs = {}        # name -> value (insertion order kept)


class _Dataset:
    def __init__(self, shape, dtype, addr):
        self.shape, self.dtype, self.addr = tuple(shape), np.dtype(dtype), addr
        self.attrs = {}


class H5Writer:
    """Streaming writer of a classic-format HDF5 file.  Paths are '/'-separated; intermediate groups
    are created on demand.  Use as a context manager or call close()."""

    def __init__(self, path):
        self.path = path
        self.f = open(path, "wb")
        self.f.write(b"\0" * SUPERBLOCK_SIZE)
        self.end = SUPERBLOCK_SIZE
        self.root = _Group()
        self.closed = False

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _node(self, path, create=True):
        node = self.root
        for part in [p for p in path.split("/") if p]:
            nxt = node.members.get(part)
            if nxt is None:
                if not create:
                    raise KeyError(path)
                nxt = node.members[part] = _Group()
            node = nxt
        return node

    def exists(self, path):
        try:
            self._node(path, create=False)
            return True
        except (KeyError, AttributeError):
            return False

    def create_group(self, path):
        """Opens or creates a group; returns True when it was created (OpenGroup's stat)."""
        created = not self.exists(path)
        g = self._node(path)
        if not isinstance(g, _Group):
            raise ValueError(f"{path} is a dataset")
        return created

    def set_attr(self, path, name, value):
        self._node(path).attrs[name] = value

    def create_dataset(self, path, data):
        """Writes data (numeric array, C order) at the end of the file now; the object header follows at
        close."""
        parent, _, name = path.rstrip("/").rpartition("/")
        g = self._node(parent)
        if name in g.members:
            raise ValueError(f"{path} exists")
        arr = np.asarray(data)
        if arr.dtype.kind == "i" and arr.dtype.itemsize == 8 and (arr.size == 0 or np.abs(arr).max() < 2**31):
            arr = arr.astype(np.int32)             # Fortran default integer
        arr = np.ascontiguousarray(arr, dtype=arr.dtype.newbyteorder("<"))
        _datatype(arr.dtype)                       # refuse unsupported types before writing anything
        addr = UNDEF
        if arr.nbytes:
            self.end += -self.end % 8
            addr = self.end
            self.f.seek(addr)
            arr.tofile(self.f)
            self.end += arr.nbytes
        g.members[name] = _Dataset(arr.shape, arr.dtype, addr)
        return g.members[name]

    # -- metadata at close -------------------------------------------------------------------
    def _layout_group(self, g):
        """Sizes and addresses of a group's heap, symbol-table nodes and B-tree nodes; then its
        members' (depth first); then its object header."""
        names = sorted(n.encode("ascii") for n in g.members)
        heap = bytearray(8)                        # offset 0: the empty name (leftmost B-tree key)
        g.name_off = {}
        for n in names:
            g.name_off[n] = len(heap)
            heap += _pad8(n + b"\0")
        g.heap_data = bytes(heap) + struct.pack("<QQ", 1, 16)    # one free block (16 bytes), last
        g.heap_addr = self._alloc(32 + len(g.heap_data))
        # symbol-table nodes of up to 2*LEAF_K members, B-tree levels of up to 2*NODE_K children
        g.snods = [names[i:i + 2 * LEAF_K] for i in range(0, len(names), 2 * LEAF_K)]
        g.snod_addr = [self._alloc(SNOD_SIZE) for _ in g.snods]
        # each B-tree level: list of nodes; a node = list of (child address, last name in child)
        level = [(a, s[-1]) for a, s in zip(g.snod_addr, g.snods)]
        g.tree = []
        while True:
            nodes = [level[i:i + 2 * NODE_K] for i in range(0, len(level), 2 * NODE_K)] or [[]]
            addrs = [self._alloc(TREE_SIZE) for _ in nodes]
            g.tree.append((nodes, addrs))
            if len(nodes) == 1:
                break
            level = [(a, n[-1][1]) for a, n in zip(addrs, nodes)]
        g.btree_addr = g.tree[-1][1][0]
        for name in sorted(g.members):
            m = g.members[name]
            if isinstance(m, _Group):
                self._layout_group(m)
            else:
                m.header = self._header(m, [(MSG_FILL, 1, _fill()), (MSG_DATATYPE, 1, _datatype(m.dtype)),
                                            (MSG_DATASPACE, 0, _dataspace(m.shape)),
                                            (MSG_LAYOUT, 1, _layout(m.shape, m.dtype.itemsize, m.addr))])
        g.header = self._header(g, [(MSG_STAB, 0, struct.pack("<QQ", g.btree_addr, g.heap_addr))])

    def _header(self, obj, msgs):
        msgs = msgs + [(MSG_ATTRIBUTE, 0, _attribute(k, v)) for k, v in obj.attrs.items()]
        obj.oh = _object_header(msgs)
        obj.oh_addr = self._alloc(len(obj.oh))
        return obj.oh

    def _alloc(self, size):
        self.end += -self.end % 8
        a = self.end
        self.end += size
        return a

    def _write_group(self, g):
        w = self.f
        w.seek(g.heap_addr)
        w.write(b"HEAP" + struct.pack("<B3xQQQ", 0, len(g.heap_data), len(g.heap_data) - 16, g.heap_addr + 32))
        w.write(g.heap_data)
        for addr, names in zip(g.snod_addr, g.snods):
            ent = b""
            for n in names:
                m = g.members[n.decode("ascii")]
                if isinstance(m, _Group):    # cache type 1: the member group's B-tree and heap
                    ent += struct.pack("<QQII", g.name_off[n], m.oh_addr, 1, 0) + struct.pack("<QQ", m.btree_addr,
                                                                                              m.heap_addr)
                else:
                    ent += struct.pack("<QQII", g.name_off[n], m.oh_addr, 0, 0) + b"\0" * 16
            w.seek(addr)
            w.write((b"SNOD" + struct.pack("<BBH", 1, 0, len(names)) + ent).ljust(SNOD_SIZE, b"\0"))
        for lev, (nodes, addrs) in enumerate(g.tree):
            left = b""                                   # the leftmost key: the empty name
            for i, (node, addr) in enumerate(zip(nodes, addrs)):
                lsib = addrs[i - 1] if i > 0 else UNDEF
                rsib = addrs[i + 1] if i + 1 < len(addrs) else UNDEF
                body = struct.pack("<Q", g.name_off.get(left, 0))
                for child, last in node:
                    body += struct.pack("<QQ", child, g.name_off[last])
                if node:
                    left = node[-1][1]
                w.seek(addr)
                w.write((b"TREE" + struct.pack("<BBHQQ", 0, lev, len(node), lsib, rsib) + body).ljust(TREE_SIZE, b"\0"))
        for name in sorted(g.members):
            m = g.members[name]
            if isinstance(m, _Group):
                self._write_group(m)
            else:
                w.seek(m.oh_addr)
                w.write(m.oh)
        w.seek(g.oh_addr)
        w.write(g.oh)

    def close(self):
        if self.closed:
            return
        self._layout_group(self.root)
        self._write_group(self.root)
        r = self.root
        sb = SIGNATURE + struct.pack("<8B", 0, 0, 0, 0, 0, 8, 8, 0) + struct.pack("<HHI", LEAF_K, NODE_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, self.end, UNDEF)
        sb += struct.pack("<QQII", 0, r.oh_addr, 1, 0) + struct.pack("<QQ", r.btree_addr, r.heap_addr)
        assert len(sb) == SUPERBLOCK_SIZE
        self.f.seek(0)
        self.f.write(sb)
        self.f.truncate(self.end)
        self.f.close()
        self.closed = True


# -- reader ------------------------------------------------------------------------------------
class _Reader:
    def __init__(self, path):
        self.b = open(path, "rb").read()
        for sb in (0, 512, 1024, 2048, 4096):      # a user block shifts the superblock by a power of 2
            if self.b[sb:sb + 8] == SIGNATURE:
                break
        else:
            raise ValueError(f"{path}: no HDF5 superblock")
        if self.b[sb + 8] != 0 or self.b[sb + 13] != 8 or self.b[sb + 14] != 8:
            raise ValueError(f"{path}: only version-0 superblocks with 8-byte offsets and lengths are read")
        self.base = struct.unpack_from("<Q", self.b, sb + 24)[0]
        self.root_oh = struct.unpack_from("<Q", self.b, sb + 64)[0]

    def u(self, fmt, addr):
        return struct.unpack_from(fmt, self.b, self.base + addr)

    def messages(self, addr):
        ver, _, n, _, size = self.u("<BBHII", addr)
        if ver != 1:
            raise ValueError(f"object header version {ver} at {addr} is not read")
        out, p = [], addr + 16
        end = p + size
        while p < end and len(out) < n:
            t, sz, fl = self.u("<HHB", p)
            out.append((t, self.base + p + 8, sz))
            p += 8 + sz
        return out

    def datatype(self, p):
        cv, b0, b1, b2, size = struct.unpack_from("<4BI", self.b, p)
        cls = cv & 0x0F
        if cls == 1:
            return np.dtype(f"<f{size}")
        if cls == 0:
            return np.dtype(f"<{'i' if b0 & 0x08 else 'u'}{size}")
        if cls == 3:
            return np.dtype(f"S{size}")
        raise ValueError(f"datatype class {cls} is not read")

    def dataspace(self, p):
        ver, rank, flags = struct.unpack_from("<3B", self.b, p)
        if ver == 1:
            q = p + 8
        elif ver == 2:
            if struct.unpack_from("<B", self.b, p + 3)[0] == 2:   # null dataspace
                return None
            q = p + 4
        else:
            raise ValueError(f"dataspace version {ver} is not read")
        return tuple(struct.unpack_from(f"<{rank}Q", self.b, q)) if rank else ()

    def attribute(self, p):
        ver, _, nlen, dlen, slen = struct.unpack_from("<BBHHH", self.b, p)
        if ver != 1:
            raise ValueError(f"attribute version {ver} is not read")
        q = p + 8
        name = self.b[q:q + nlen].rstrip(b"\0").decode("ascii")
        q += nlen + (-nlen % 8)
        dt = self.datatype(q)
        q += dlen + (-dlen % 8)
        shape = self.dataspace(q)
        q += slen + (-slen % 8)
        n = int(np.prod(shape)) if shape else 1
        val = np.frombuffer(self.b, dtype=dt, count=n, offset=q).reshape(shape)
        if dt.kind == "S":
            val = val.item().rstrip(b"\0").decode("ascii") if val.ndim == 0 else val
        elif val.ndim == 0:
            val = val.item()
        return name, val

    def layout(self, p, shape, dt):
        ver = self.b[p]
        if ver in (1, 2):
            rank, cls = struct.unpack_from("<BB", self.b, p + 1)
            if cls != 1:
                raise ValueError(f"layout class {cls} is not read")
            return struct.unpack_from("<Q", self.b, p + 8)[0]
        if ver == 3:
            cls = self.b[p + 1]
            if cls == 1:
                return struct.unpack_from("<Q", self.b, p + 2)[0]
            if cls == 0:
                size = struct.unpack_from("<H", self.b, p + 2)[0]
                return ("compact", p + 4, size)
            raise ValueError(f"layout class {cls} is not read")
        raise ValueError(f"layout version {ver} is not read")

    def group(self, btree, heap):
        hsig, _, _, _, daddr = self.u("<4sB3xQQQ", heap)
        if hsig != b"HEAP":
            raise ValueError("bad local heap")
        out = {}

        def name_at(off):
            s = self.base + daddr + off
            return self.b[s:self.b.index(b"\0", s)].decode("ascii")

        def walk(addr):
            sig, typ, lev, n = self.u("<4sBBH", addr)
            if sig != b"TREE" or typ != 0:
                raise ValueError("bad group B-tree node")
            for i in range(n):
                child = self.u("<Q", addr + 24 + 8 + 16 * i)[0]
                if lev > 0:
                    walk(child)
                    continue
                ssig, _, _, ns = self.u("<4sBBH", child)
                if ssig != b"SNOD":
                    raise ValueError("bad symbol-table node")
                for j in range(ns):
                    noff, oh = self.u("<QQ", child + 8 + 40 * j)
                    out[name_at(noff)] = self.object(oh)

        walk(btree)
        return out

    def object(self, addr):
        msgs = self.messages(addr)
        attrs, shape, dt, lay, stab = {}, None, None, None, None
        for t, p, sz in msgs:
            if t == MSG_ATTRIBUTE:
                k, v = self.attribute(p)
                attrs[k] = v
            elif t == MSG_DATASPACE:
                shape = self.dataspace(p)
            elif t == MSG_DATATYPE:
                dt = self.datatype(p)
            elif t == MSG_LAYOUT:
                lay = p
            elif t == MSG_STAB:
                stab = struct.unpack_from("<QQ", self.b, p)
        if stab is not None:
            node = Node(self.group(*stab))
            node.attrs = attrs
            return node
        where = self.layout(lay, shape, dt)
        n = int(np.prod(shape)) if shape else 1
        if isinstance(where, tuple):
            data = np.frombuffer(self.b, dtype=dt, count=n, offset=where[1])
        elif where == UNDEF:
            data = np.zeros(n, dtype=dt)
        else:
            data = np.frombuffer(self.b, dtype=dt, count=n, offset=self.base + where)
        arr = data.reshape(shape).copy()
        return Dataset(arr, attrs)


class Node(dict):
    """A group read back: members by name, attributes in .attrs."""
    attrs = {}


class Dataset(np.ndarray):
    """A dataset read back: the array, attributes in .attrs."""

    def __new__(cls, arr, attrs):
        obj = np.asarray(arr).view(cls)
        obj.attrs = attrs
        return obj

    def __array_finalize__(self, obj):
        self.attrs = getattr(obj, "attrs", {})


def read(path):
    """Reads a classic-format HDF5 file into nested dicts (Node) of arrays (Dataset)."""
    r = _Reader(path)
    return r.object(r.root_oh)


# -- the Lionbolt results schema ---------------------------------------------------------------
ATTR_PROBTYPE = "problem_type"
ATTR_OBJTYPE = "object_type"
GROUP_MESH = "mesh"
DATASET_R, DATASET_CONNECTIVITY, DATASET_OFFSET, DATASET_VOLS = ("global_nodes", "connectivity", "offset",
                                                                 "element_volumes")
ATTR_NUMMATS_M, ATTR_NUMELS, ATTR_NUMSD, ATTR_NUMKG = ("number_of_materials", "number_of_elements",
                                                       "number_of_spatial_dofs", "number_of_global_nodes")
GROUP_MAT2SD = "material_to_spatial_dof"
ATTR_NUMANGLES, DATASET_ANGWEIGHTS, DATASET_ABSCISSAE = "number_of_angular_dofs", "angular_weights", "abscissae"
ATTR_NUMENERGIES, DATASET_EGRID = "number_of_energy_dofs", "energy_grid"
IS_PARTICLE = "particle"
GROUP_FL, GROUP_FL_UNC = "fluence", "uncollided_fluence"
GROUP_ANG_FL, GROUP_ANG_FL_UNC = "angular_fluence", "uncollided_angular_fluence"
PATTERN_ENERGY, PATTERN_ANGLE, PATTERN_MATERIALS = "energy_", "angle_", "material_"
PATTERN_DEP = "_deposition"
DATASET_EDEP, DATASET_DDEP, DATASET_CDEP = "energy", "dose", "charge"


def element_volumes(mesh):
    x = mesh.rg[mesh.node]                                   # [NE, 4, 3]
    return np.abs(np.linalg.det(x[:, 1:] - x[:, :1])) / 6.0


class ResultsFile:
    """The reference's results writer (LionboltHDF5.f90) over H5Writer, with an active group as the
    reference's HDF5Tree keeps one.  Group and angle indices are 1-based in the names, as written by
    the reference (energy_1 ... energy_G, angle_1 ... angle_NI, material_1 ... material_Nm)."""

    def __init__(self, path):
        self.h5 = H5Writer(path)
        self.active = ""

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def close(self):
        self.h5.close()

    def _p(self, *parts):
        return "/".join(p for p in (self.active,) + parts if p)

    def write_problem_type(self, probtype):
        """WriteProblemTypeH5 (:77-84): attribute of the active group."""
        self.h5.set_attr(self.active, ATTR_PROBTYPE, probtype)

    def open_particle(self, particle, nolc=False):
        """OpenParticleH5 (:15-46): the particle's group in the root, tagged object_type = particle when
        created."""
        name = particle.strip() if nolc else particle.strip().lower()
        self.active = ""
        if self.h5.create_group(name):
            self.h5.set_attr(name, ATTR_OBJTYPE, IS_PARTICLE)
        self.active = name

    def close_particle(self, particle=None):
        """CloseParticleH5 (:48-75): back to the root."""
        self.active = ""

    def write_mesh(self, mesh, slab=False):
        """WriteMeshH5 (:86-202): the mesh group in the root, one-based connectivity."""
        NE, NENK, NK, Nm = mesh.NE, mesh.NENK, mesh.NN, mesh.Nm
        g = GROUP_MESH
        self.h5.create_group(g)
        self.h5.set_attr(g, ATTR_PROBTYPE, "slab" if slab else "general")
        for k, v in ((ATTR_NUMMATS_M, Nm), (ATTR_NUMELS, NE), (ATTR_NUMSD, NENK), (ATTR_NUMKG, NK)):
            self.h5.set_attr(g, k, np.int32(v))
        self.h5.create_dataset(f"{g}/{DATASET_CONNECTIVITY}", (mesh.node.reshape(-1) + 1).astype(np.int32))
        self.h5.create_dataset(f"{g}/{DATASET_OFFSET}", (4 * np.arange(NE + 1)).astype(np.int32))
        self.h5.create_dataset(f"{g}/{DATASET_R}", np.asarray(mesh.rg, dtype=np.float64))
        self.h5.create_group(f"{g}/{GROUP_MAT2SD}")
        sdof_mat = np.repeat(np.asarray(mesh.mat), 4)
        for m in range(Nm):
            sd = np.flatnonzero(sdof_mat == m) + 1 if Nm > 1 else np.arange(1, NENK + 1)
            self.h5.create_dataset(f"{g}/{GROUP_MAT2SD}/{PATTERN_MATERIALS}{m + 1}", sd.astype(np.int32))
        self.h5.create_dataset(f"{g}/{DATASET_VOLS}", element_volumes(mesh))

    def append_ordinates(self, w, k):
        """AppendOrdinatesH5 (:204-219): k is [NI, 3] (the reference's k(3, NI))."""
        w = np.asarray(w, dtype=np.float64)
        self.h5.set_attr(self.active, ATTR_NUMANGLES, np.int32(w.size))
        self.h5.create_dataset(self._p(DATASET_ANGWEIGHTS), w)
        self.h5.create_dataset(self._p(DATASET_ABSCISSAE), np.asarray(k, dtype=np.float64).reshape(w.size, 3))

    def append_energy_grid(self, E):
        """AppendEnergyGridH5 (:221-231): G + 1 group bounds."""
        E = np.asarray(E, dtype=np.float64)
        self.h5.set_attr(self.active, ATTR_NUMENERGIES, np.int32(E.size - 1))
        self.h5.create_dataset(self._p(DATASET_EGRID), E)

    def append_spatial_array(self, name, x, g=None):
        """AppendSpatialArray (:233-272): name/energy_<g> when g is given (1-based), else a dataset."""
        x = np.asarray(x, dtype=np.float64)
        if g is None:
            self.h5.create_dataset(self._p(name), x)
        else:
            self.h5.create_group(self._p(name))
            self.h5.create_dataset(self._p(name, f"{PATTERN_ENERGY}{g}"), x)

    def append_angular_fluence(self, x, NENK, uncollided, g):
        """AppendAngularFluence (:274-336): x is angle-major [NI * NENK]; one dataset per angle."""
        x = np.asarray(x, dtype=np.float64).reshape(-1)
        grp = self._p(GROUP_ANG_FL_UNC if uncollided else GROUP_ANG_FL, f"{PATTERN_ENERGY}{g}")
        self.h5.create_group(grp)
        for i in range(x.size // NENK):
            self.h5.create_dataset(f"{grp}/{PATTERN_ANGLE}{i + 1}", x[i * NENK:(i + 1) * NENK])

    def add_dataset(self, name, x):
        """AddDataset in the active group (the deposition tallies, Main.f90:807-821)."""
        self.h5.create_dataset(self._p(name), np.asarray(x))


def write_results(path, mesh, w, k, flux, dose=None, particle="photon", energy_grid=None, uncollided=None,
                  problem_type="general", slab=False):
    """A results file laid out as Main.f90 writes it (:118, :178, :213-231, :449-469, :807-821): the
    problem type, the mesh, the particle group with its energy grid, ordinates and per-group fluence
    (and uncollided fluence of the groups where it is non-zero), and the dose deposition in the root.
    flux is [G, NENK]; uncollided is [G, NENK] or None."""
    flux = np.asarray(flux, dtype=np.float64)
    with ResultsFile(path) as out:
        out.write_problem_type(problem_type)
        out.write_mesh(mesh, slab=slab)
        out.open_particle(particle)
        if energy_grid is not None:
            out.append_energy_grid(energy_grid)
        out.append_ordinates(w, k)
        for g in range(flux.shape[0]):
            out.append_spatial_array(GROUP_FL, flux[g], g + 1)
            if uncollided is not None and np.any(uncollided[g]):
                out.append_spatial_array(GROUP_FL_UNC, uncollided[g], g + 1)
        out.close_particle(particle)
        if dose is not None:
            out.add_dataset(DATASET_DDEP + PATTERN_DEP, np.asarray(dose, dtype=np.float64))
    return path


__all__ = ["H5Writer", "ResultsFile", "read", "write_results", "element_volumes"]
