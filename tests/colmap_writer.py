"""Writes COLMAP binary scenes (sparse/0/{cameras,images,points3D}.bin) and
binary PPM images for the loader tests, following COLMAP's documented binary
format (the layout the reference's readers parse, src/io/data_io.cpp:79-200):

cameras.bin   u64 count; per camera i32 id, i32 model, u64 width, u64 height,
              model params as doubles (PINHOLE = model 1: fx, fy, cx, cy)
images.bin    u64 count; per image i32 id, 4 doubles qvec (w, x, y, z), 3 doubles
              tvec, i32 camera id, NUL-terminated name, u64 n2d, n2d x
              (double x, double y, i64 point3D id)
points3D.bin  u64 count; per point u64 id, 3 doubles xyz, 3 u8 rgb, double error,
              u64 track length, track x (i32 image id, i32 point2D index)
"""
import os
import struct
import zlib

import numpy as np


def write_ppm(path, rgb):
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    with open(path, "wb") as f:
        f.write(b"P6\n# written by the loader tests\n%d %d\n255\n" % (rgb.shape[1], rgb.shape[0]))
        f.write(rgb.tobytes())


def quaternion_to_matrix(q):
    w, x, y, z = np.asarray(q, dtype=np.float64) / np.linalg.norm(q)
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)],
    ])


def matrix_to_quaternion(R):
    """Unit quaternion (w, x, y, z) of a rotation matrix (Shepperd's method)."""
    R = np.asarray(R, dtype=np.float64)
    t = np.trace(R)
    if t > 0:
        s = 2.0 * np.sqrt(1.0 + t)
        q = [0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s]
    elif R[0, 0] > R[1, 1] and R[0, 0] > R[2, 2]:
        s = 2.0 * np.sqrt(1.0 + R[0, 0] - R[1, 1] - R[2, 2])
        q = [(R[2, 1] - R[1, 2]) / s, 0.25 * s, (R[0, 1] + R[1, 0]) / s, (R[0, 2] + R[2, 0]) / s]
    elif R[1, 1] > R[2, 2]:
        s = 2.0 * np.sqrt(1.0 + R[1, 1] - R[0, 0] - R[2, 2])
        q = [(R[0, 2] - R[2, 0]) / s, (R[0, 1] + R[1, 0]) / s, 0.25 * s, (R[1, 2] + R[2, 1]) / s]
    else:
        s = 2.0 * np.sqrt(1.0 + R[2, 2] - R[0, 0] - R[1, 1])
        q = [(R[1, 0] - R[0, 1]) / s, (R[0, 2] + R[2, 0]) / s, (R[1, 2] + R[2, 1]) / s, 0.25 * s]
    q = np.array(q)
    return q / np.linalg.norm(q)


def write_scene(root, width, height, fx, fy, cx, cy, views, points, colors, image_ext=".jpg", model=1,
                camera_id=1, n2d=3):
    """views: list of dicts {name, qvec, tvec, image (HxWx3 u8 or None)}. Images
    are written as images/<stem>.ppm (the pre-decoded form of <name>)."""
    sparse = os.path.join(root, "sparse", "0")
    image_dir = os.path.join(root, "images")
    os.makedirs(sparse, exist_ok=True)
    os.makedirs(image_dir, exist_ok=True)
    with open(os.path.join(sparse, "cameras.bin"), "wb") as f:
        f.write(struct.pack("<Q", 1))
        f.write(struct.pack("<iiQQ", camera_id, model, width, height))
        f.write(struct.pack("<4d", fx, fy, cx, cy))
    with open(os.path.join(sparse, "images.bin"), "wb") as f:
        f.write(struct.pack("<Q", len(views)))
        for k, v in enumerate(views):
            f.write(struct.pack("<i", k + 1))
            f.write(struct.pack("<4d", *v["qvec"]))
            f.write(struct.pack("<3d", *v["tvec"]))
            f.write(struct.pack("<i", v.get("camera_id", 1)))
            f.write(v["name"].encode() + b"\0")
            f.write(struct.pack("<Q", n2d))
            for j in range(n2d):
                f.write(struct.pack("<ddq", 1.5 * j, 2.5 * j, j if j % 2 == 0 else -1))
            if v.get("image") is not None:
                stem = os.path.splitext(v["name"])[0]
                write_ppm(os.path.join(image_dir, stem + ".ppm"), v["image"])
    with open(os.path.join(sparse, "points3D.bin"), "wb") as f:
        f.write(struct.pack("<Q", len(points)))
        for k, (p, c) in enumerate(zip(points, colors)):
            f.write(struct.pack("<Q", k))
            f.write(struct.pack("<3d", *[float(x) for x in p]))
            f.write(struct.pack("<3B", *[int(x) for x in c]))
            f.write(struct.pack("<d", 0.5))
            track = k % 3
            f.write(struct.pack("<Q", track))
            for j in range(track):
                f.write(struct.pack("<ii", j + 1, j))


def decode_png(path):
    """8-bit RGB, non-interlaced PNG with filter 0 rows (what the library writes)."""
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, chunks = 8, {}
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        (crc,) = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(kind + body) & 0xFFFFFFFF
        chunks.setdefault(kind, b"")
        chunks[kind] += body
        pos += 12 + n
    w, h, depth, colour, _, _, interlace = struct.unpack(">IIBBBBB", chunks[b"IHDR"])
    assert (depth, colour, interlace) == (8, 2, 0)
    raw = zlib.decompress(chunks[b"IDAT"])
    rows = np.frombuffer(raw, np.uint8).reshape(h, 1 + 3 * w)
    assert (rows[:, 0] == 0).all()
    assert b"IEND" in chunks
    return rows[:, 1:].reshape(h, w, 3)
