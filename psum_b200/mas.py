"""PSuM's MAS ("multi-array-set") checkpoint format, for particle groups and
node fields of this library.

A MAS file is a sequence of blocks (src/serialization/mas.hpp:130-161,
mas_file::writeData), each

    "#MAS!#"                       magic string (6 bytes)
    int32 key_len, int32 type_len, int32 shape_len
    key (key_len bytes), type name (type_len bytes)
    shape_len x uint64 dimensions
    the elements, row-major, native little-endian

where the type name is PSuM's MATLAB-style name of the element type
(foundation.hpp:91-113: double, single, int64, uint64, int32, uint32, int16,
uint16, int8, uint8, logical, char).  A block whose key starts with '!' is
masked (mas_file::smashData writes '!' over the key's first byte) and is
skipped when the file is read; writing a key that is already present is an
error (MAS_STRICT_NAME_CHECKING 2, mas.hpp:17-21).

The composite objects are stored as PSuM's serializers lay them out:

    simple_grid<D>          name.lower, name.upper (double, D x 1), name.cells (int32, D x 1)
                            (simple_grid.hpp:428-433)
    device_field            name.location (int32, 1 x 1; 3 = node centred), name.grid.*,
                            name.content.device (char), name.content.content (double, n x 1)
                            (device_field.hpp:326-331, device_array.hpp:188-204)
    particle_group          name.data.device (char), and per tag of the particle struct
                            name.data.content.position (double, n x D x 1),
                            name.data.content.velocity (double, n x 3 x 1)
                            (particle_group.hpp:271-274, device_vector.hpp:293-308,
                            tag_sl.hpp:61-92, container_sl.hpp:96-108)

A group is written as its stored particles (compacted after a sort or a
fused step); an invalid particle is written with NaN position components,
as PSuM writes its invalid slots, and load() drops it the same way.  The
".device" strings follow PSuM's "[#k]<device name>" form.
"""
import os
import struct

import numpy as np

MAGIC = b"#MAS!#"
NODE_CENTERED = 3   # field::var_loc::nodeCentered (field/foundation.hpp:14-19)

# numpy dtype <-> PSuM (MATLAB) type name
_TYPES = [
    (np.dtype(np.float64), "double"), (np.dtype(np.float32), "single"),
    (np.dtype(np.int64), "int64"), (np.dtype(np.uint64), "uint64"),
    (np.dtype(np.int32), "int32"), (np.dtype(np.uint32), "uint32"),
    (np.dtype(np.int16), "int16"), (np.dtype(np.uint16), "uint16"),
    (np.dtype(np.int8), "int8"), (np.dtype(np.uint8), "uint8"),
    (np.dtype(np.bool_), "logical"), (np.dtype("S1"), "char"),
]
_NAME_OF = {dt: name for dt, name in _TYPES}
_DTYPE_OF = {name: dt for dt, name in _TYPES}


class MasDuplicateBlockError(RuntimeError):
    """A block with this key already exists (mas_duplicate_block_error)."""


class MasBlockInfo:
    __slots__ = ("name", "type", "shape", "size", "position")

    def __init__(self, name, type_, shape, position):
        self.name, self.type, self.shape, self.position = name, type_, tuple(shape), position
        self.size = int(np.prod(shape, dtype=np.int64)) if len(shape) else 1

    def __repr__(self):
        return f"MasBlockInfo({self.name!r}, {self.type!r}, {self.shape})"


class MasFile:
    """mas_file (mas.hpp:53-440): mode "auto" opens or creates, "replace"
    starts an empty file, "quick" opens an existing file without reading its
    block heads."""

    def __init__(self, path, mode="auto"):
        self.path = os.fspath(path)
        self.heads = []
        if not os.path.exists(self.path):
            if mode == "quick":
                raise FileNotFoundError(f"Error: file not found: {self.path}")
            parent = os.path.dirname(self.path)
            if parent:
                os.makedirs(parent, exist_ok=True)
            open(self.path, "wb").close()
        if mode == "auto":
            self.read_head()
        elif mode == "replace":
            self.clear()
        elif mode != "quick":
            raise ValueError(f"unknown mode {mode!r}")

    def clear(self):
        open(self.path, "wb").close()
        self.heads = []

    def _find(self, key, type_="*"):
        return [h for h in self.heads if h.name == key and (type_ == "*" or h.type == type_)]

    def keys(self):
        return [h.name for h in self.heads]

    def write(self, key, data, shape=None):
        """writeData: data is an array (or str / bytes for a char block);
        shape defaults to (len, 1) for 1-D data, as PSuM's vector save does."""
        if not key:
            raise ValueError("Error: key can't be empty")
        if key[0] == "!":
            raise ValueError("Error: key can't start with '!'")
        if isinstance(data, str):
            data = data.encode()
        if isinstance(data, (bytes, bytearray)):
            arr = np.frombuffer(bytes(data), dtype="S1")
        else:
            arr = np.asarray(data)
            if arr.dtype.kind == "S":
                arr = arr.view("S1")
        dt = arr.dtype
        if dt not in _NAME_OF:
            raise TypeError(f"unsupported element type {dt}")
        if shape is None:
            shape = (arr.size, 1) if arr.ndim <= 1 else arr.shape
        shape = tuple(int(s) for s in shape)
        if int(np.prod(shape, dtype=np.int64)) != arr.size:
            raise ValueError(f"shape {shape} does not hold {arr.size} elements")
        if self._find(key):
            raise MasDuplicateBlockError(f"Error: block already exists: {key}")
        name = _NAME_OF[dt].encode()
        kb = key.encode()
        with open(self.path, "ab") as f:
            pos = f.tell()
            f.write(MAGIC)
            f.write(struct.pack("<iii", len(kb), len(name), len(shape)))
            f.write(kb)
            f.write(name)
            f.write(struct.pack(f"<{len(shape)}Q", *shape))
            f.write(np.ascontiguousarray(arr).astype(dt.newbyteorder("<"), copy=False).tobytes())
        self.heads.append(MasBlockInfo(key, _NAME_OF[dt], shape, pos))

    def read_head(self):
        """readHead: the unmasked blocks, in file order."""
        heads = []
        with open(self.path, "rb") as f:
            data = f.read()
        p = 0
        while p < len(data):
            pos = p
            if data[p:p + 6] != MAGIC:
                raise ValueError("Error: magic string mismatch.")
            p += 6
            if p + 12 > len(data):
                raise ValueError("Error: failed to read block information.")
            kl, tl, sl = struct.unpack_from("<iii", data, p)
            p += 12
            key = data[p:p + kl].decode(errors="replace")
            p += kl
            type_ = data[p:p + tl].decode()
            p += tl
            shape = struct.unpack_from(f"<{sl}Q", data, p)
            p += 8 * sl
            if type_ not in _DTYPE_OF:
                raise ValueError(f"Error: unknown block type {type_!r}")
            nbytes = int(np.prod(shape, dtype=np.int64)) * _DTYPE_OF[type_].itemsize
            if p + nbytes > len(data):
                raise ValueError(f"Error: incomplete MAS block: {key}")
            p += nbytes
            if not key.startswith("!"):
                heads.append(MasBlockInfo(key, type_, shape, pos))
        self.heads = heads
        return heads

    def read(self, key, type_="*"):
        """readData: (info, array shaped like the block) or (None, None)."""
        if not self._find(key, type_):
            self.read_head()
        found = self._find(key, type_)
        if not found:
            return None, None
        h = found[0]
        with open(self.path, "rb") as f:
            f.seek(h.position + 6 + 12 + len(h.name.encode()) + len(h.type) + 8 * len(h.shape))
            dt = _DTYPE_OF[h.type]
            raw = f.read(h.size * dt.itemsize)
        if len(raw) != h.size * dt.itemsize:
            raise ValueError(f"Error: incomplete MAS block: {key}")
        return h, np.frombuffer(raw, dtype=dt.newbyteorder("<")).reshape(h.shape).astype(dt)

    def smash(self, key, type_="*"):
        """smashData: mask every matching block ('!' over its key's first byte)."""
        found = self._find(key, type_)
        with open(self.path, "r+b") as f:
            for h in found:
                f.seek(h.position + 6 + 12)
                f.write(b"!")
        self.heads = [h for h in self.heads if h not in found]
        return bool(found)

    def replace(self, key, data, shape=None):
        """replaceData: mask the block of the same key and type, write it again."""
        probe = np.asarray(data.encode() if isinstance(data, str) else data)
        type_ = "char" if probe.dtype.kind == "S" or isinstance(data, (str, bytes)) else _NAME_OF.get(probe.dtype, "*")
        self.smash(key, type_)
        self.write(key, data, shape)

    def read_string(self, key):
        _, arr = self.read(key, "char")
        if arr is None:
            raise KeyError(key)
        return arr.reshape(-1).tobytes().decode()


def _device_string():
    """PSuM's "[#k]<device name>" (k = index among devices of that name)."""
    try:
        import torch
        if torch.cuda.is_available():
            i = torch.cuda.current_device()
            name = torch.cuda.get_device_name(i)
            k = sum(1 for j in range(i) if torch.cuda.get_device_name(j) == name)
            return f"[#{k}]{name}"
    except Exception:
        pass
    return "[#0]host"


def save_grid(fp, name, grid):
    """simple_grid save (simple_grid.hpp:428-433)."""
    d = grid.dim
    fp.write(name + ".lower", np.asarray(grid.lower[:d], np.float64))
    fp.write(name + ".upper", np.asarray(grid.upper[:d], np.float64))
    fp.write(name + ".cells", np.asarray(grid.cells[:d], np.int32))


def load_grid(fp, name):
    """(lower, upper, cells) of a saved simple_grid."""
    out = []
    for part, dt in ((".lower", np.float64), (".upper", np.float64), (".cells", np.int32)):
        h, arr = fp.read(name + part)
        if arr is None:
            raise KeyError(name + part)
        if len(h.shape) != 2 or h.shape[1] != 1:
            raise ValueError(f"Error: block '{name + part}' cannot be loaded as vector.")
        out.append(arr.reshape(-1).astype(dt))
    return tuple(out)


def save_node_field(fp, name, grid, values):
    """device_field<nodeCentered> save (device_field.hpp:326-331): location,
    grid and content (device_array: .device and .content)."""
    v = _host(values).astype(np.float64, copy=False).reshape(-1)
    if v.size != grid.n_nodes:
        raise ValueError(f"field has {v.size} values, the grid {grid.n_nodes} nodes")
    fp.write(name + ".location", np.asarray([NODE_CENTERED], np.int32), (1, 1))
    save_grid(fp, name + ".grid", grid)
    fp.write(name + ".content.device", _device_string())
    fp.write(name + ".content.content", v)


def load_node_field(fp, name, grid=None):
    """Values of a saved node field (checked against grid when given)."""
    _, loc = fp.read(name + ".location")
    if loc is None:
        raise KeyError(name + ".location")
    if int(loc.reshape(-1)[0]) != NODE_CENTERED:
        raise ValueError(f"Error: block '{name}' has location {int(loc.reshape(-1)[0])} which cannot be loaded "
                         f"into a field of location {NODE_CENTERED}.")
    lower, upper, cells = load_grid(fp, name + ".grid")
    h, v = fp.read(name + ".content.content")
    if v is None:
        raise KeyError(name + ".content.content")
    v = v.reshape(-1)
    if v.size != int(np.prod(cells.astype(np.int64) + 1)):
        raise ValueError(f"Error: block '{name}' has a content size which does not match its grid.")
    if grid is not None and (list(cells) != list(grid.cells[:grid.dim])
                             or not np.allclose(lower, grid.lower[:grid.dim])
                             or not np.allclose(upper, grid.upper[:grid.dim])):
        raise ValueError(f"Error: block '{name}' was saved on another grid")
    return v


def save_particle_group(fp, name, ctx, species):
    """particle_group save (particle_group.hpp:271-274): the stored
    particles' FP64 positions (n x dim x 1) and velocities (n x 3 x 1)."""
    pos, vel = ctx.get_state(species)          # (dim, n), (3, n) FP64 host arrays
    n = pos.shape[1]
    fp.write(name + ".data.device", _device_string())
    fp.write(name + ".data.content.position", np.ascontiguousarray(pos.T), (n, pos.shape[0], 1))
    fp.write(name + ".data.content.velocity", np.ascontiguousarray(vel.T), (n, vel.shape[0], 1))
    return n


def load_particle_group(fp, name, ctx, species):
    """particle_group load (particle_group.hpp:277-283): clear and insert.
    Particles with a non-finite position become invalid, as in PSuM."""
    hp, pos = fp.read(name + ".data.content.position")
    hv, vel = fp.read(name + ".data.content.velocity")
    if pos is None or vel is None:
        raise KeyError(name + ".data.content")
    if len(hp.shape) != 3 or hp.shape[1] != ctx.dim or len(hv.shape) != 3 or hv.shape[0] != hp.shape[0]:
        raise ValueError(f"Error: block '{name}' cannot be loaded as a particle group of this context.")
    n = hp.shape[0]
    pos = np.ascontiguousarray(pos.reshape(n, hp.shape[1]).T.astype(np.float64))
    v3 = np.zeros((3, n))
    v3[: hv.shape[1]] = vel.reshape(n, hv.shape[1]).T[:3]
    ctx.load(species, pos, v3)
    return n


def _host(x):
    try:
        import torch
        if isinstance(x, torch.Tensor):
            return x.detach().cpu().numpy()
    except Exception:
        pass
    return np.asarray(x)
