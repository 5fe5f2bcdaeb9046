"""Reader for the reference's precomputed operators: MATLAB v7.3 MAT-files.

``precompute_collision_operator.m:52-61`` builds a ``GeneralCollisionTensor`` and saves it, with its
``SpectralBasis`` and ``ScatteringKernel``, by ``save(..., '-v7.3')``; the solvers load it back
(``tutorial_stress_relaxation.m:36-51``) and read ``TensorObj.{R_tensor, gaunt_labels, gaunt_vals,
ic_map}``.  ``load_collision_tensor`` reads those four arrays (and the scalar properties) into the
layout ``CollisionOperator`` takes, so a precomputed file drives the GPU operator directly.

A v7.3 MAT-file is an HDF5 file behind a 512-byte user block.  ``MatFile`` reads the subset of
HDF5 MATLAB writes -- the version-0 superblock, version-1 object headers, symbol-table groups (v1
B-trees of group nodes over a local heap), and datasets stored compact, contiguous, or chunked (v1
B-tree of chunks, deflate filter) with IEEE float, fixed-point, string and object-reference
element types -- following the published HDF5 file-format specification.

MATLAB arrays are column-major and HDF5 datasets row-major: a MATLAB array of size [a, b, c] is
an HDF5 dataset of dims (c, b, a).  ``MatFile.array`` returns it with MATLAB's shape (Fortran
order).

Class instances (MCOS objects) are saved as a 1x1 ``uint32`` reference record
[0xDD000000, ndims, dims..., object ids..., class id] at the variable's place; their property
values live in one cell array, the ``FileWrapper__`` object under ``/#subsystem#/MCOS``, whose
first cell is a metadata blob: a u32 version, the number of names, eight region offsets, the
NUL-separated names (class and property names), then the regions (class table: package and class
name per class; saveobj property blocks; object table: class, saveobj block, property block and
dependency id per object; property blocks).  A property block lists (name index, kind, value)
triplets: kind 0 names a string, kind 1 points at cell ``value + 2`` of the FileWrapper cell
array, kind 2 holds the value itself.
"""
from __future__ import annotations

import zlib
from dataclasses import dataclass, field

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
_UNDEF = (1 << 64) - 1
_OBJ_REF_TAG = 0xDD000000


class MatFormatError(ValueError):
    """The file uses an HDF5 or MAT-file feature this reader does not handle, or is damaged."""


@dataclass
class MatObject:
    """A MATLAB class instance: its class name and its saved property values."""

    class_name: str
    props: dict = field(default_factory=dict)

    def __getitem__(self, name):
        return self.props[name]


@dataclass
class MatOpaque:
    """A value this reader does not decode (function handles, structs): its MATLAB class only."""

    class_name: str


class MatFile:
    """One v7.3 MAT-file, read into memory."""

    def __init__(self, path: str):
        with open(path, "rb") as fh:
            self.buf = fh.read()
        sb = self.buf.find(SIGNATURE)
        if sb < 0 or sb % 512:
            raise MatFormatError(f"{path}: no HDF5 superblock (not a v7.3 MAT-file)")
        if self.buf[sb + 8] != 0:
            raise MatFormatError(f"superblock version {self.buf[sb + 8]} not handled")
        if self.buf[sb + 13] != 8 or self.buf[sb + 14] != 8:
            raise MatFormatError("only 8-byte offsets and lengths are handled")
        p = sb + 24
        self.base = self._u(p, 8)
        # base, free-space, end-of-file and driver-info addresses, then the root symbol-table entry
        self.root = self._u(p + 32 + 8, 8)
        self._fw = None

    # ------------------------------------------------------------------ primitives
    def _u(self, pos: int, n: int) -> int:
        return int.from_bytes(self.buf[pos:pos + n], "little")

    def _at(self, addr: int) -> int:
        p = self.base + addr
        if not 0 <= p < len(self.buf):
            raise MatFormatError(f"address {addr} outside the file")
        return p

    # ------------------------------------------------------------------ object headers
    def messages(self, header: int) -> list:
        """(type, payload) of every message of the version-1 object header at ``header``."""
        p = self._at(header)
        if self.buf[p] != 1:
            raise MatFormatError(f"object header version {self.buf[p]} not handled")
        n_msgs = self._u(p + 2, 2)
        blocks = [(p + 16, self._u(p + 8, 4))]
        out = []
        while blocks and len(out) < n_msgs:
            q, length = blocks.pop(0)
            end = q + length
            while q + 8 <= end and len(out) < n_msgs:
                mtype, msize = self._u(q, 2), self._u(q + 2, 2)
                data = self.buf[q + 8:q + 8 + msize]
                if mtype == 0x10:  # continuation block
                    blocks.append((self._at(int.from_bytes(data[0:8], "little")), int.from_bytes(data[8:16], "little")))
                out.append((mtype, data))
                q += 8 + msize
        return out

    # ------------------------------------------------------------------ groups
    def _heap_string(self, heap: int, offset: int) -> str:
        p = self._at(heap)
        if self.buf[p:p + 4] != b"HEAP":
            raise MatFormatError("bad local heap")
        data = self._at(self._u(p + 24, 8)) + offset
        return self.buf[data:self.buf.index(b"\x00", data)].decode()

    def _group_tree(self, node: int, heap: int, out: dict):
        p = self._at(node)
        if self.buf[p:p + 4] != b"TREE" or self.buf[p + 4] != 0:
            raise MatFormatError("bad group B-tree node")
        level, used = self.buf[p + 5], self._u(p + 6, 2)
        q = p + 24 + 8  # node header, then key 0
        for _ in range(used):
            child = self._u(q, 8)
            q += 16  # child pointer and the key after it
            if level:
                self._group_tree(child, heap, out)
                continue
            s = self._at(child)
            if self.buf[s:s + 4] != b"SNOD":
                raise MatFormatError("bad symbol-table node")
            e = s + 8
            for _ in range(self._u(s + 6, 2)):
                out[self._heap_string(heap, self._u(e, 8))] = self._u(e + 8, 8)
                e += 40

    def children(self, header: int) -> dict:
        """name -> object-header address of the members of the group at ``header``."""
        for mtype, data in self.messages(header):
            if mtype == 0x11:  # symbol table: B-tree and local heap
                out: dict = {}
                self._group_tree(int.from_bytes(data[0:8], "little"), int.from_bytes(data[8:16], "little"), out)
                return out
        raise MatFormatError("not a group")

    def resolve(self, path: str) -> int:
        addr = self.root
        for part in [x for x in path.split("/") if x]:
            members = self.children(addr)
            if part not in members:
                raise KeyError(path)
            addr = members[part]
        return addr

    # ------------------------------------------------------------------ datatypes, attributes
    @staticmethod
    def _dataspace(data: bytes) -> tuple:
        version, ndim = data[0], data[1]
        off = 8 if version == 1 else 4
        return tuple(int.from_bytes(data[off + 8 * i:off + 8 * i + 8], "little") for i in range(ndim))

    @staticmethod
    def _datatype(data: bytes) -> np.dtype:
        cls, bits, size = data[0] & 0x0F, data[1], int.from_bytes(data[4:8], "little")
        if bits & 1:
            raise MatFormatError("big-endian data not handled")
        if cls == 1:
            return np.dtype(f"<f{size}")
        if cls == 0:
            return np.dtype(f"<{'i' if bits & 0x08 else 'u'}{size}")
        if cls == 3:
            return np.dtype(f"S{size}")
        if cls == 7:  # object reference: an address
            return np.dtype("<u8")
        raise MatFormatError(f"datatype class {cls} not handled")

    def attributes(self, header: int) -> dict:
        out = {}
        for mtype, data in self.messages(header):
            if mtype != 0x0C:
                continue
            version = data[0]
            nlen, tlen, slen = (int.from_bytes(data[i:i + 2], "little") for i in (2, 4, 6))
            pad = (lambda n: (n + 7) // 8 * 8) if version == 1 else (lambda n: n)
            q = 8
            name = data[q:q + nlen].rstrip(b"\x00").decode()
            q += pad(nlen)
            try:
                dtype = self._datatype(data[q:q + tlen])
            except MatFormatError:  # e.g. variable-length strings inside function-handle workspaces
                continue
            q += pad(tlen)
            sdata = data[q:q + slen]
            q += pad(slen)
            dims = self._dataspace(sdata) if len(sdata) > 1 and sdata[1] else ()
            count = int(np.prod(dims)) if dims else 1
            val = np.frombuffer(data[q:q + count * dtype.itemsize], dtype, count)
            if dtype.kind == "S":
                out[name] = b"".join(val.tolist()).rstrip(b"\x00").decode()
            else:
                out[name] = val.reshape(dims) if dims else val[0]
        return out

    # ------------------------------------------------------------------ datasets
    @staticmethod
    def _filter_ids(data: bytes) -> list:
        version, n = data[0], data[1]
        q = 8 if version == 1 else 2
        ids = []
        for _ in range(n):
            fid = int.from_bytes(data[q:q + 2], "little")
            named = version == 1 or fid >= 256
            name_len = int.from_bytes(data[q + 2:q + 4], "little") if named else 0
            q += 4 if named else 2
            n_vals = int.from_bytes(data[q + 2:q + 4], "little")
            q += 4
            q += ((name_len + 7) // 8 * 8) if version == 1 else name_len
            q += 4 * n_vals + (4 if version == 1 and n_vals % 2 else 0)
            ids.append(fid)
        return ids

    def dataset(self, where) -> np.ndarray:
        """The elements of a dataset (a path or an object-header address) in HDF5 shape."""
        header = self.resolve(where) if isinstance(where, str) else int(where)
        dims = dtype = layout = None
        filters: list = []
        for mtype, data in self.messages(header):
            if mtype == 0x01:
                dims = self._dataspace(data)
            elif mtype == 0x03:
                dtype = self._datatype(data)
            elif mtype == 0x08:
                layout = data
            elif mtype == 0x0B:
                filters = self._filter_ids(data)
        if dims is None or dtype is None or layout is None:
            raise MatFormatError("not a dataset")
        if layout[0] != 3:
            raise MatFormatError(f"data layout version {layout[0]} not handled")
        if set(filters) - {1}:
            raise MatFormatError(f"filters {filters} not handled (deflate only)")
        count = int(np.prod(dims)) if dims else 1
        nbytes = count * dtype.itemsize
        kind = layout[1]
        if kind == 0:  # compact: the data sits in the message
            raw = layout[4:4 + int.from_bytes(layout[2:4], "little")]
        elif kind == 1:  # contiguous
            a = int.from_bytes(layout[2:10], "little")
            raw = b"" if a == _UNDEF else self.buf[self._at(a):self._at(a) + nbytes]
        elif kind == 2:  # chunked
            ndim = layout[2]
            tree = int.from_bytes(layout[3:11], "little")
            cdims = tuple(int.from_bytes(layout[11 + 4 * i:15 + 4 * i], "little") for i in range(ndim - 1))
            return self._chunked(tree, dims, cdims, dtype, 1 in filters)
        else:
            raise MatFormatError(f"layout class {kind} not handled")
        if len(raw) < nbytes:  # storage never allocated: the fill value (zero)
            return np.zeros(dims, dtype)
        return np.frombuffer(raw, dtype, count).reshape(dims).copy()

    def _chunked(self, tree: int, dims: tuple, cdims: tuple, dtype: np.dtype, deflate: bool) -> np.ndarray:
        out = np.zeros(dims, dtype)
        nd = len(dims)
        key = 8 + 8 * (nd + 1)  # chunk size, filter mask, nd + 1 offsets
        csize = int(np.prod(cdims)) * dtype.itemsize

        def walk(node):
            p = self._at(node)
            if self.buf[p:p + 4] != b"TREE" or self.buf[p + 4] != 1:
                raise MatFormatError("bad chunk B-tree node")
            level, used = self.buf[p + 5], self._u(p + 6, 2)
            q = p + 24
            for _ in range(used):
                size, mask = self._u(q, 4), self._u(q + 4, 4)
                offs = [self._u(q + 8 + 8 * i, 8) for i in range(nd)]
                child = self._u(q + key, 8)
                if level:
                    walk(child)
                else:
                    raw = self.buf[self._at(child):self._at(child) + size]
                    if deflate and not mask & 1:
                        raw = zlib.decompress(raw)
                    if len(raw) != csize:
                        raise MatFormatError("chunk size mismatch")
                    chunk = np.frombuffer(raw, dtype).reshape(cdims)
                    dst = tuple(slice(o, min(o + c, d)) for o, c, d in zip(offs, cdims, dims))
                    out[dst] = chunk[tuple(slice(0, s.stop - s.start) for s in dst)]
                q += key + 8

        walk(tree)
        return out

    # ------------------------------------------------------------------ MATLAB values
    def array(self, where) -> np.ndarray:
        """A numeric dataset with MATLAB's shape (Fortran order)."""
        return np.asfortranarray(self.dataset(where).T)

    def variables(self) -> list:
        return [n for n in self.children(self.root) if not n.startswith("#")]

    def load(self, name: str):
        """A top-level variable: numeric arrays, char, logical, cells and MCOS objects."""
        return self._value(self.resolve(name))

    def _value(self, header: int):
        attrs = self.attributes(header)
        cls = attrs.get("MATLAB_class", "")
        if attrs.get("MATLAB_empty", 0):
            dims = self.dataset(header).ravel()
            return np.zeros(tuple(int(d) for d in dims), dtype=np.float64)
        if "MATLAB_object_decode" in attrs and cls != "FileWrapper__":
            ref = self.dataset(header).T.ravel()
            return self._object_from_ref(ref, cls)
        if cls == "cell":
            refs = self.dataset(header).T
            return [self._value(int(r)) for r in refs.ravel(order="F")]
        if cls in ("char",):
            codes = self.dataset(header).T
            return "".join(chr(int(c)) for c in codes.ravel(order="F"))
        if cls == "logical":
            return self.array(header).astype(bool)
        if cls in ("double", "single", "int8", "uint8", "int16", "uint16", "int32", "uint32", "int64", "uint64"):
            arr = self.array(header)
            # an object nested in another object's properties: a bare uint32 reference record
            if cls == "uint32" and arr.ndim == 2 and arr.shape[1] == 1 and arr.shape[0] >= 6 \
                    and int(arr[0, 0]) == _OBJ_REF_TAG:
                return self._object_from_ref(arr.ravel(), cls)
            return arr
        return MatOpaque(cls)

    # ------------------------------------------------------------------ MCOS objects
    def _filewrapper(self):
        if self._fw is None:
            cells = self.dataset("/#subsystem#/MCOS").ravel()
            meta = self.dataset(int(cells[0])).ravel().tobytes()
            n_names = int.from_bytes(meta[4:8], "little")
            offs = [int.from_bytes(meta[8 + 4 * i:12 + 4 * i], "little") for i in range(8)]
            names = [s.decode() for s in meta[40:offs[0]].split(b"\x00")[:n_names]]

            def region(i):
                return np.frombuffer(meta[offs[i]:offs[i + 1]], "<u4").astype(np.int64)

            classes = region(0).reshape(-1, 4)  # package name, class name, 0, 0 (row 0 unused)
            objects = region(2).reshape(-1, 6)  # class, 0, 0, saveobj block, property block, dependency
            self._fw = dict(cells=cells, names=names, classes=classes, objects=objects,
                            saved=self._blocks(region(1)), props=self._blocks(region(3)))
        return self._fw

    @staticmethod
    def _blocks(words: np.ndarray) -> list:
        """Property blocks: block 0 is empty; each block is n, then n (name, kind, value) triplets,
        padded to a multiple of 8 bytes."""
        blocks, q = [[]], 2
        while q < words.size:
            n = int(words[q])
            trip = words[q + 1:q + 1 + 3 * n].reshape(-1, 3)
            blocks.append([tuple(int(x) for x in t) for t in trip])
            q += 1 + 3 * n
            q += q % 2
        return blocks

    def _object_from_ref(self, ref: np.ndarray, cls: str):
        ref = [int(x) for x in ref]
        if not ref or ref[0] != _OBJ_REF_TAG:
            return MatOpaque(cls)
        ndims = ref[1]
        dims = ref[2:2 + ndims]
        count = int(np.prod(dims))
        ids = ref[2 + ndims:2 + ndims + count]
        objs = [self.object(i) for i in ids]
        return objs[0] if count == 1 else objs

    def object(self, obj_id: int) -> MatObject:
        """Object ``obj_id`` (1-based) of the file's MCOS table with its properties."""
        fw = self._filewrapper()
        cls_i, _, _, saved_i, prop_i, _ = (int(x) for x in fw["objects"][obj_id])
        cname = fw["names"][int(fw["classes"][cls_i][1]) - 1]
        pkg = int(fw["classes"][cls_i][0])
        if pkg:
            cname = fw["names"][pkg - 1] + "." + cname
        obj = MatObject(cname)
        for block in (fw["saved"][saved_i] if saved_i else [], fw["props"][prop_i] if prop_i else []):
            for name_i, kind, value in block:
                pname = fw["names"][name_i - 1]
                if kind == 0:
                    obj.props[pname] = fw["names"][value - 1]
                elif kind == 1:
                    obj.props[pname] = self._value(int(fw["cells"][value + 2]))
                else:
                    obj.props[pname] = value
        return obj


@dataclass
class CollisionTensorFile:
    """The operator arrays of a saved ``GeneralCollisionTensor`` (src/GeneralCollisionTensor.m:9-12)."""

    K_max: int
    L_max: int
    R: np.ndarray  # [K x K x K x N_L], Fortran order, K = K_max + 1
    labels: np.ndarray  # [N_G x 3] float64, 1-based
    vals: np.ndarray  # [N_G] float64
    ic_map: np.ndarray  # [N_G] float64, 1-based
    alpha: float | None  # ScatteringKernel.alpha, when saved

    @property
    def K(self) -> int:
        return self.K_max + 1

    @property
    def N_Q(self) -> int:
        return (self.L_max + 1) ** 2

    def sorted_for_contraction(self):
        """(labels, vals, ic_map) in stable sortrows([ic_map, q1]) order, the order the reference's
        contraction callers pass to the MEX kernels (benchmark_collision_contraction_scaling.m:82-85)."""
        o = np.lexsort((self.labels[:, 0], self.ic_map))
        return np.ascontiguousarray(self.labels[o]), self.vals[o].copy(), self.ic_map[o].copy()

    def operator(self, device: int = 0):
        """A device-resident ``CollisionOperator`` over this file's arrays (contraction order)."""
        from .operator import CollisionOperator

        labels, vals, ic_map = self.sorted_for_contraction()
        return CollisionOperator(labels, vals, ic_map, self.R, self.N_Q, self.K, device=device)


def load_collision_tensor(path: str, variable: str = "TensorObj") -> CollisionTensorFile:
    """Read the ``GeneralCollisionTensor`` saved as ``variable`` (precompute_collision_operator.m:61)."""
    mf = MatFile(path)
    obj = mf.load(variable)
    if not isinstance(obj, MatObject) or obj.class_name != "GeneralCollisionTensor":
        raise MatFormatError(f"{variable} is not a GeneralCollisionTensor")
    p = obj.props
    R = np.asfortranarray(p["R_tensor"], dtype=np.float64)
    labels = np.ascontiguousarray(p["gaunt_labels"], dtype=np.float64)
    n_g = labels.shape[0]
    vals = np.asarray(p["gaunt_vals"], dtype=np.float64).reshape(n_g)
    ic_map = np.asarray(p["ic_map"], dtype=np.float64).reshape(n_g)
    kern = p.get("Kernel")
    alpha = None
    if isinstance(kern, MatObject) and "alpha" in kern.props:
        alpha = float(np.asarray(kern.props["alpha"]).ravel()[0])
    return CollisionTensorFile(K_max=int(np.asarray(p["K_max"]).ravel()[0]), L_max=int(np.asarray(p["L_max"]).ravel()[0]),
                               R=R, labels=labels, vals=vals, ic_map=ic_map, alpha=alpha)
