"""On-disk formats of the experiment drivers: PLY point clouds and meshes.

Same file layouts as mpm_exps/engine/mesh_io.py: particle dumps are binary
little-endian PLY files with one `vertex` element of float x, y, z
(`write_point_cloud_packed`, :68-80) or x, y, z, vel_x, vel_y, vel_z
(`write_point_cloud`, :49-65); meshes are PLY files with `vertex` and
`face` elements (`load_mesh`, :14-33).  The reader here is self-contained
(ascii, binary little- and big-endian; scalar and list properties), so no
PLY package is needed.
"""
import numpy as np

_TYPES = {
    "char": "i1", "int8": "i1", "uchar": "u1", "uint8": "u1", "short": "i2", "int16": "i2",
    "ushort": "u2", "uint16": "u2", "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4",
    "float": "f4", "float32": "f4", "double": "f8", "float64": "f8",
}


def _header(n, names):
    lines = ["ply", "format binary_little_endian 1.0", "comment Created by taichi", "element vertex %d" % n]
    lines += ["property float %s" % nm for nm in names]
    return ("\n".join(lines) + "\nend_header\n").encode()


def write_point_cloud_packed(fn, pos, num_particles=None):
    """Particle positions (n x 3 float32, row-major) as a binary PLY file:
    what dump_states writes (mpm_solver.py:1776-1780)."""
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    n = len(pos) if num_particles is None else int(num_particles)
    if pos.ndim != 2 or pos.shape[1] != 3 or len(pos) != n:
        raise ValueError("write_point_cloud_packed: expected %d x 3 positions, got %s" % (n, pos.shape))
    with open(fn, "wb") as f:
        f.write(_header(n, ["x", "y", "z"]))
        f.write(pos.tobytes())


def write_point_cloud(fn, pos_and_vel):
    """Positions and velocities (n x 6 float32) as a binary PLY file."""
    a = np.ascontiguousarray(pos_and_vel, dtype=np.float32)
    if a.ndim != 2 or a.shape[1] != 6:
        raise ValueError("write_point_cloud: expected n x 6 values, got %s" % (a.shape,))
    with open(fn, "wb") as f:
        f.write(_header(len(a), ["x", "y", "z", "vel_x", "vel_y", "vel_z"]))
        f.write(a.tobytes())


def _parse_header(f):
    if f.readline().strip() != b"ply":
        raise ValueError("not a PLY file")
    fmt, elems = None, []
    while True:
        line = f.readline()
        if not line:
            raise ValueError("PLY header without end_header")
        tok = line.decode("ascii", "replace").split()
        if not tok or tok[0] in ("comment", "obj_info"):
            continue
        if tok[0] == "end_header":
            break
        if tok[0] == "format":
            fmt = tok[1]
        elif tok[0] == "element":
            elems.append((tok[1], int(tok[2]), []))
        elif tok[0] == "property":
            if not elems:
                raise ValueError("PLY property before any element")
            if tok[1] == "list":
                elems[-1][2].append((tok[4], _TYPES[tok[2]], _TYPES[tok[3]]))
            else:
                elems[-1][2].append((tok[2], _TYPES[tok[1]], None))
    if fmt not in ("ascii", "binary_little_endian", "binary_big_endian"):
        raise ValueError("unsupported PLY format %r" % fmt)
    return fmt, elems


def read_ply(fn):
    """{element name: {property name: array}}; list properties become a
    list of arrays (or an n x k array when every list has k entries)."""
    out = {}
    with open(fn, "rb") as f:
        fmt, elems = _parse_header(f)
        if fmt == "ascii":
            words = f.read().split()
            pos = 0
            for name, n, props in elems:
                cols = {p[0]: [] for p in props}
                for _ in range(n):
                    for pname, t, it in props:
                        if it is None:
                            cols[pname].append(words[pos])
                            pos += 1
                        else:
                            k = int(words[pos])
                            cols[pname].append(np.array(words[pos + 1:pos + 1 + k], dtype=it))
                            pos += 1 + k
                out[name] = {p[0]: (np.array(cols[p[0]], dtype=p[1]) if p[2] is None else _lists(cols[p[0]]))
                             for p in props}
            return out
        end = "<" if fmt == "binary_little_endian" else ">"
        data = f.read()
    off = 0
    for name, n, props in elems:
        if all(p[2] is None for p in props):
            dt = np.dtype([(p[0], end + p[1]) for p in props])
            rec = np.frombuffer(data, dtype=dt, count=n, offset=off)
            off += n * dt.itemsize
            out[name] = {p[0]: rec[p[0]].astype(p[1]) for p in props}
            continue
        fast = _fixed_lists(data, off, n, props, end)
        if fast is not None:  # every list of the element has the same length
            out[name], off = fast
            continue
        cols = {p[0]: [] for p in props}
        for _ in range(n):
            for pname, t, it in props:
                if it is None:
                    v = np.frombuffer(data, dtype=end + t, count=1, offset=off)[0]
                    off += np.dtype(t).itemsize
                    cols[pname].append(v)
                else:
                    k = int(np.frombuffer(data, dtype=end + t, count=1, offset=off)[0])
                    off += np.dtype(t).itemsize
                    cols[pname].append(np.frombuffer(data, dtype=end + it, count=k, offset=off).astype(it))
                    off += k * np.dtype(it).itemsize
        out[name] = {p[0]: (np.array(cols[p[0]], dtype=p[1]) if p[2] is None else _lists(cols[p[0]]))
                     for p in props}
    return out


def _fixed_lists(data, off, n, props, end):
    """Vectorized read of an element whose lists all have the length of the
    first record's (triangle faces): ({name: array}, new offset), or None."""
    if n == 0:
        return {p[0]: np.zeros((0,), dtype=p[1]) if p[2] is None else np.zeros((0, 0), dtype=p[2])
                for p in props}, off
    fields, pos = [], off
    for pname, t, it in props:  # list lengths from the first record
        if it is None:
            fields.append((pname, end + t))
            pos += np.dtype(t).itemsize
        else:
            k = int(np.frombuffer(data, dtype=end + t, count=1, offset=pos)[0])
            fields.append(("_n_" + pname, end + t))
            fields.append((pname, end + it, (k,)))
            pos += np.dtype(t).itemsize + k * np.dtype(it).itemsize
    dt = np.dtype(fields)
    if off + n * dt.itemsize > len(data):
        return None
    rec = np.frombuffer(data, dtype=dt, count=n, offset=off)
    for pname, t, it in props:
        if it is not None and not np.all(rec["_n_" + pname] == dt[pname].shape[0]):
            return None
    return {p[0]: rec[p[0]].astype(p[1] if p[2] is None else p[2]) for p in props}, off + n * dt.itemsize


def _lists(v):
    if v and all(len(x) == len(v[0]) for x in v):
        return np.stack(v)
    return v


def load_particles_only(fn):
    """n x 3 positions of the first element of a PLY file (load_states)."""
    el = next(iter(read_ply(fn).values()))
    x, y, z = el["x"], el["y"], el["z"]
    if not len(x) == len(y) == len(z):
        raise ValueError("ragged x, y, z")
    return np.stack([x, y, z], axis=1)


def load_mesh(fn, scale=1, offset=(0, 0, 0)):
    """Triangles (n x 9 float32: a, b, c corners) of a triangle mesh,
    scaled per axis and offset (mesh_io.py:14-33)."""
    if isinstance(scale, (int, float)):
        scale = (scale, scale, scale)
    ply = read_ply(fn)
    v = np.stack([ply["vertex"]["x"], ply["vertex"]["y"], ply["vertex"]["z"]], axis=1).astype(np.float64)
    faces = ply["face"].get("vertex_indices", ply["face"].get("vertex_index"))
    faces = np.asarray(faces)
    if faces.ndim != 2 or faces.shape[1] != 3:
        raise ValueError("load_mesh: only triangle faces are supported")
    v = v * np.asarray(scale, dtype=np.float64) + np.asarray(offset, dtype=np.float64)
    return v[faces].reshape(len(faces), 9).astype(np.float32)


def load_mesh_vertices_and_indices(fn):
    """Vertices with y and z swapped and the new z negated, and the flat
    triangle index list (mesh_io.py:36-46)."""
    ply = read_ply(fn)
    vx = ply["vertex"]
    vertices = np.stack([vx["x"], vx["z"], vx["y"]], axis=1)
    vertices[:, -1] *= -1
    faces = ply["face"].get("vertex_indices", ply["face"].get("vertex_index"))
    return vertices, np.concatenate([np.asarray(f).ravel() for f in faces])
