"""Texture images of XML scenes (src/gpu/DXRApp_Textures.cpp:34-40,448-537):
the host's PNG / TGA / BMP / PPM readers against images written here with an
independent encoder (Python's zlib for DEFLATE, numpy for the expected
texels), malformed files, and the texture wiring of scene flattening —
sRGB for albedo maps only, one load per resolved file, unreadable files
leaving the constant parameter in place.  GPU: an XML scene with texture
maps renders the same image as its flattened buffers uploaded directly."""

import ctypes as C
import os
import struct
import subprocess
import sys
import zlib

import numpy as np
import pytest

from test_nori_host import LIBNORI, flat, load, nori, write_hdr  # noqa: F401  (fixture)

ADAM7 = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]


@pytest.fixture(scope="module")
def img(nori):
    nori.nori_load_image.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_char_p, C.c_size_t]
    nori.nori_load_image.restype = C.c_uint64
    nori.nori_texture.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    nori.nori_texture.restype = C.c_uint64

    def read(path):
        wh = (C.c_uint32 * 2)()
        err = C.create_string_buffer(512)
        n = nori.nori_load_image(str(path).encode(), wh, None, 0, err, 512)
        if n == 0:
            raise ValueError(err.value.decode())
        out = np.zeros(n, np.uint8)
        assert nori.nori_load_image(str(path).encode(), wh, out.ctypes.data, n, err, 512) == n
        return out.reshape(wh[1], wh[0], 4)
    return read


# ---------------------------------------------------------------------------- PNG writer
def chunk(kind, data):
    return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xFFFFFFFF)


def paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = np.abs(p - a), np.abs(p - b), np.abs(p - c)
    return np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, b, c))


def filter_rows(rows, bpp, rng):
    """Forward PNG filtering of raw scanlines (list of uint8 arrays), a random
    filter type per row; returns the bytes of the filtered image."""
    out = bytearray()
    prev = np.zeros_like(rows[0], dtype=np.int32) if rows else None
    for r in rows:
        x = r.astype(np.int32)
        a = np.concatenate([np.zeros(bpp, np.int32), x[:-bpp]]) if len(x) > bpp else np.zeros_like(x)
        if len(x) > bpp:
            c = np.concatenate([np.zeros(bpp, np.int32), prev[:-bpp]])
        else:
            c = np.zeros_like(x)
        b = prev
        f = int(rng.integers(0, 5))
        y = [x, x - a, x - b, x - (a + b) // 2, x - paeth(a, b, c)][f]
        out.append(f)
        out += (y & 0xFF).astype(np.uint8).tobytes()
        prev = x
    return bytes(out)


def pack_rows(samples, depth):
    """samples: (h, w*channels) integer array -> list of packed scanlines."""
    rows = []
    for s in samples:
        if depth == 16:
            rows.append(s.astype(">u2").view(np.uint8).copy())
        elif depth == 8:
            rows.append(s.astype(np.uint8))
        else:
            per = 8 // depth
            n = (len(s) + per - 1) // per
            padded = np.zeros(n * per, np.uint32)
            padded[:len(s)] = s
            v = np.zeros(n, np.uint32)
            for k in range(per):
                v |= padded[k::per] << (8 - depth * (k + 1))
            rows.append(v.astype(np.uint8))
    return rows


def encode_png(samples, colour, depth, palette=None, trns=None, interlace=False, strategy=None, level=6,
               split=0, seed=0):
    """samples: (h, w, channels) integer array at the given bit depth."""
    h, w, ch = samples.shape
    rng = np.random.default_rng(seed)
    bpp = max(1, ch * depth // 8)
    if not interlace:
        raw = filter_rows(pack_rows(samples.reshape(h, w * ch), depth), bpp, rng)
    else:
        raw = b""
        for x0, y0, dx, dy in ADAM7:
            sub = samples[y0::dy, x0::dx]
            if sub.size:
                raw += filter_rows(pack_rows(sub.reshape(sub.shape[0], -1), depth), bpp, rng)
    if strategy is None:
        z = zlib.compress(raw, level)
    else:
        co = zlib.compressobj(level, zlib.DEFLATED, 15, 9, strategy)
        z = co.compress(raw) + co.flush()
    out = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, colour, 0, 0, int(interlace)))
    if palette is not None:
        out += chunk(b"PLTE", np.asarray(palette, np.uint8).tobytes())
    if trns is not None:
        out += chunk(b"tRNS", trns)
    pieces = [z] if not split else [z[i:i + split] for i in range(0, len(z), split)]
    for p in pieces:
        out += chunk(b"IDAT", p)
    return out + chunk(b"IEND", b"")


def expected_rgba(samples, colour, depth, palette=None, trns=None):
    s = samples.astype(np.int64)
    to8 = (lambda v: v >> 8) if depth == 16 else (lambda v: v * (255 // ((1 << depth) - 1)))
    h, w, _ = s.shape
    out = np.zeros((h, w, 4), np.int64)
    if colour == 3:
        pal = np.full((256, 4), 255, np.int64)
        pal[:, :3] = 0
        p = np.asarray(palette).reshape(-1, 3)
        pal[:len(p), :3] = p
        if trns is not None:
            pal[:len(trns), 3] = np.frombuffer(trns, np.uint8)
        out[:] = pal[s[..., 0]]
        out[s[..., 0] >= len(p)] = [0, 0, 0, 255]
    elif colour in (0, 4):
        out[..., :3] = to8(s[..., :1])
        out[..., 3] = to8(s[..., 1]) if colour == 4 else 255
        if colour == 0 and trns is not None:
            out[s[..., 0] == struct.unpack(">H", trns)[0], 3] = 0
    else:
        out[..., :3] = to8(s[..., :3])
        out[..., 3] = to8(s[..., 3]) if colour == 6 else 255
        if colour == 2 and trns is not None:
            key = np.array(struct.unpack(">HHH", trns))
            out[(s[..., :3] == key).all(-1), 3] = 0
    return out.astype(np.uint8)


PNG_CASES = []
for depth in (1, 2, 4, 8, 16):
    PNG_CASES.append((0, depth))
for depth in (1, 2, 4, 8):
    PNG_CASES.append((3, depth))
for colour in (2, 4, 6):
    for depth in (8, 16):
        PNG_CASES.append((colour, depth))


def random_png(colour, depth, w, h, seed, with_trns=True):
    rng = np.random.default_rng(seed)
    ch = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[colour]
    hi = (1 << depth) if colour != 3 else min(1 << depth, 200)
    samples = rng.integers(0, hi, (h, w, ch))
    palette = trns = None
    if colour == 3:
        n = min(1 << depth, 180)
        palette = rng.integers(0, 256, (n, 3))
        samples %= n + 2  # a few indices past the palette
        if with_trns:
            trns = rng.integers(0, 256, min(n, 7)).astype(np.uint8).tobytes()
    elif colour == 0 and with_trns:
        samples[0, 0, 0] = samples[-1, -1, 0]
        trns = struct.pack(">H", int(samples[0, 0, 0]))
    elif colour == 2 and with_trns:
        samples[1 % h, 0] = samples[0, 0]
        trns = struct.pack(">HHH", *map(int, samples[0, 0]))
    return samples, palette, trns


@pytest.mark.parametrize("colour,depth", PNG_CASES)
@pytest.mark.parametrize("interlace", [False, True])
def test_png_colour_types_and_depths(img, tmp_path, colour, depth, interlace):
    for (w, h) in [(13, 7), (1, 1), (3, 5)] if interlace else [(13, 7), (1, 1), (33, 2)]:
        samples, pal, trns = random_png(colour, depth, w, h, seed=w * 31 + h + depth)
        p = tmp_path / f"c{colour}d{depth}_{w}x{h}.png"
        p.write_bytes(encode_png(samples, colour, depth, pal, trns, interlace=interlace, seed=w + h))
        got = img(p)
        assert np.array_equal(got, expected_rgba(samples, colour, depth, pal, trns)), (w, h)


@pytest.mark.parametrize("how", ["stored", "fixed", "rle", "huffman_only", "best", "split_idat"])
def test_png_deflate_block_kinds(img, tmp_path, how):
    """Stored, fixed-Huffman, dynamic-Huffman blocks; overlapping copies (RLE
    strategy: distance 1); several IDAT chunks."""
    rng = np.random.default_rng(7)
    smooth = (np.add.outer(np.arange(40), np.arange(57)) // 3 % 256)[..., None].repeat(4, -1)
    samples = np.where(rng.random(smooth.shape) < 0.05, rng.integers(0, 256, smooth.shape), smooth)
    kw = dict(stored=dict(level=0), fixed=dict(strategy=zlib.Z_FIXED), rle=dict(strategy=zlib.Z_RLE),
              huffman_only=dict(strategy=zlib.Z_HUFFMAN_ONLY), best=dict(level=9),
              split_idat=dict(split=97))[how]
    p = tmp_path / f"{how}.png"
    p.write_bytes(encode_png(samples, 6, 8, **kw))
    assert np.array_equal(img(p), samples.astype(np.uint8))


def test_png_large_stored_blocks(img, tmp_path):
    """An image bigger than one stored block (65535 bytes)."""
    rng = np.random.default_rng(2)
    samples = rng.integers(0, 256, (150, 200, 3))
    p = tmp_path / "big.png"
    p.write_bytes(encode_png(samples, 2, 8, level=0))
    assert np.array_equal(img(p)[..., :3], samples.astype(np.uint8))


def valid_png(seed=0):
    samples = np.random.default_rng(seed).integers(0, 256, (9, 11, 4))
    return encode_png(samples, 6, 8), samples


@pytest.mark.parametrize("mutate,msg", [
    (lambda b: b[:len(b) // 2], "runs past the file"),
    (lambda b: b[:-12], "ends before IEND"),
    (lambda b: b[:8] + b[8:33].replace(b"\x08\x06", b"\x08\x05", 1) + b[33:], "colour type"),
    (lambda b: b[:8] + b[8:33].replace(b"\x08\x06\x00\x00\x00", b"\x08\x06\x00\x00\x02", 1) + b[33:],
     "interlace"),
    (lambda b: b.replace(b"IDAT", b"IDAX"), "zlib header"),
])
def test_png_malformed(img, tmp_path, mutate, msg):
    p = tmp_path / "bad.png"
    p.write_bytes(mutate(valid_png()[0]))
    with pytest.raises(ValueError, match=msg):
        img(p)


def test_png_bad_filter_and_truncated_data(img, tmp_path):
    samples = np.zeros((4, 4, 4), np.int64)
    raw = b"".join(bytes([5]) + bytes(16) for _ in range(4))  # filter type 5 does not exist
    out = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", 4, 4, 8, 6, 0, 0, 0))
    p = tmp_path / "f5.png"
    p.write_bytes(out + chunk(b"IDAT", zlib.compress(raw)) + chunk(b"IEND", b""))
    with pytest.raises(ValueError, match="filter type"):
        img(p)
    short = b"".join(bytes([0]) + bytes(16) for _ in range(3))  # one row missing
    p.write_bytes(out + chunk(b"IDAT", zlib.compress(short)) + chunk(b"IEND", b""))
    with pytest.raises(ValueError, match="shorter than the image"):
        img(p)
    long = b"".join(bytes([0]) + bytes(16) for _ in range(9))  # more data than 4 rows
    p.write_bytes(out + chunk(b"IDAT", zlib.compress(long)) + chunk(b"IEND", b""))
    with pytest.raises(ValueError, match="more image data"):
        img(p)
    del samples


def test_png_fuzz_never_crashes(tmp_path):
    """Random byte corruption of valid PNGs: every file decodes or raises, in a
    child process so that a crash fails this test instead of the run."""
    files = []
    rng = np.random.default_rng(11)
    for k in range(150):
        b = bytearray(valid_png(k % 5)[0] if k % 2 else encode_png(
            np.random.default_rng(k).integers(0, 16, (13, 7, 1)), 3, 4, palette=np.zeros((16, 3)), interlace=True))
        for _ in range(int(rng.integers(1, 6))):
            b[int(rng.integers(8, len(b)))] = int(rng.integers(0, 256))
        if k % 7 == 0:
            b = b[:int(rng.integers(8, len(b)))]
        p = tmp_path / f"fz{k}.png"
        p.write_bytes(bytes(b))
        files.append(str(p))
    code = f"""
import ctypes as C, sys
L = C.CDLL({LIBNORI!r})
L.nori_load_image.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_char_p, C.c_size_t]
L.nori_load_image.restype = C.c_uint64
wh = (C.c_uint32 * 2)(); err = C.create_string_buffer(256); ok = 0
for f in sys.argv[1:]:
    n = L.nori_load_image(f.encode(), wh, None, 0, err, 256)
    if n: buf = (C.c_uint8 * n)(); L.nori_load_image(f.encode(), wh, buf, n, err, 256); ok += 1
print(ok)
"""
    r = subprocess.run([sys.executable, "-c", code, *files], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr


# ---------------------------------------------------------------------------- TGA / BMP / PNM
def test_tga(img, tmp_path):
    rng = np.random.default_rng(3)
    px = rng.integers(0, 256, (5, 7, 4)).astype(np.uint8)
    px[2, 1:6] = px[2, 1]  # a run for the RLE encoder

    def header(kind, bits, top):
        return bytes([0, 0, kind]) + bytes(9) + struct.pack("<HH", 7, 5) + bytes([bits, 0x20 if top else 0])

    bgra = px[..., [2, 1, 0, 3]]
    # uncompressed 32-bit, top-down
    (tmp_path / "a.tga").write_bytes(header(2, 32, True) + bgra.tobytes())
    assert np.array_equal(img(tmp_path / "a.tga"), px)
    # uncompressed 24-bit, bottom-up
    (tmp_path / "b.tga").write_bytes(header(2, 24, False) + bgra[::-1, :, :3].tobytes())
    exp = px.copy()
    exp[..., 3] = 255
    assert np.array_equal(img(tmp_path / "b.tga"), exp)
    # run-length 32-bit, top-down: raw packets and run packets
    flat_px = bgra.reshape(-1, 4)
    body = bytearray()
    i = 0
    while i < len(flat_px):
        j = i
        while j + 1 < len(flat_px) and j - i < 127 and (flat_px[j + 1] == flat_px[i]).all():
            j += 1
        if j > i:
            body += bytes([0x80 | (j - i)]) + flat_px[i].tobytes()
            i = j + 1
        else:
            body += bytes([0]) + flat_px[i].tobytes()
            i += 1
    (tmp_path / "c.tga").write_bytes(header(10, 32, True) + bytes(body))
    assert np.array_equal(img(tmp_path / "c.tga"), px)
    # 8-bit grey
    (tmp_path / "d.tga").write_bytes(header(3, 8, True) + px[..., 0].tobytes())
    g = np.repeat(px[..., :1], 3, -1)
    assert np.array_equal(img(tmp_path / "d.tga")[..., :3], g)
    (tmp_path / "e.tga").write_bytes(header(10, 32, True) + bytes(body[:-3]))
    with pytest.raises(ValueError, match="truncated"):
        img(tmp_path / "e.tga")


@pytest.mark.parametrize("bits,top", [(24, False), (32, True), (24, True)])
def test_bmp(img, tmp_path, bits, top):
    rng = np.random.default_rng(bits)
    W, H = 5, 3
    px = rng.integers(0, 256, (H, W, 4)).astype(np.uint8)
    bp = bits // 8
    stride = (W * bp + 3) & ~3
    rows = px[:, :, [2, 1, 0, 3]][:, :, :bp]
    data = b"".join(r.tobytes() + bytes(stride - W * bp) for r in (rows if top else rows[::-1]))
    hdr = b"BM" + struct.pack("<IHHI", 54 + len(data), 0, 0, 54)
    info = struct.pack("<IiiHHIIiiII", 40, W, -H if top else H, 1, bits, 0, len(data), 2835, 2835, 0, 0)
    (tmp_path / "a.bmp").write_bytes(hdr + info + data)
    exp = px.copy()
    if bits == 24:
        exp[..., 3] = 255
    assert np.array_equal(img(tmp_path / "a.bmp"), exp)


def test_pnm(img, tmp_path):
    rng = np.random.default_rng(5)
    rgb = rng.integers(0, 256, (4, 6, 3)).astype(np.uint8)
    (tmp_path / "a.ppm").write_bytes(b"P6\n# comment\n6 4\n255\n" + rgb.tobytes())
    got = img(tmp_path / "a.ppm")
    assert np.array_equal(got[..., :3], rgb) and (got[..., 3] == 255).all()
    low = rng.integers(0, 101, (4, 6)).astype(np.uint8)
    (tmp_path / "b.pgm").write_bytes(b"P5 6 4 100\n" + low.tobytes())
    got = img(tmp_path / "b.pgm")
    exp = ((low.astype(np.int64) * 255 + 50) // 100).astype(np.uint8)
    assert np.array_equal(got[..., 0], exp) and np.array_equal(got[..., 2], exp)


def test_unsupported_formats(img, tmp_path):
    (tmp_path / "a.jpg").write_bytes(b"\xff\xd8\xff\xe0" + bytes(100))
    with pytest.raises(ValueError, match="JPEG"):
        img(tmp_path / "a.jpg")
    (tmp_path / "a.xyz").write_bytes(b"hello world")
    with pytest.raises(ValueError, match="unknown image format"):
        img(tmp_path / "a.xyz")
    with pytest.raises(ValueError, match="cannot open"):
        img(tmp_path / "missing.png")


# ---------------------------------------------------------------------------- scenes with textures
def write_obj_uv(path, v, uv, f):
    with open(path, "w") as o:
        for p in v:
            o.write(f"v {p[0]:.7g} {p[1]:.7g} {p[2]:.7g}\n")
        for t in uv:
            o.write(f"vt {t[0]:.7g} {t[1]:.7g}\n")
        for t in f:
            o.write("f " + " ".join(f"{i + 1}/{i + 1}" for i in t) + "\n")


TEX_XML = """<?xml version="1.0"?>
<scene>
  <string name="envmap" value="sky.hdr"/>
  <float name="envmapScale" value="0.3"/>
  <integrator type="path_mis"><integer name="maxDepth" value="8"/></integrator>
  <camera type="perspective">
    <float name="fov" value="45"/>
    <transform name="toWorld"><lookat origin="0, 1.6, 4.5" target="0, 0.4, 0" up="0, 1, 0"/></transform>
    <integer name="width" value="64"/><integer name="height" value="48"/>
  </camera>
  <sampler type="independent"><integer name="sampleCount" value="4"/></sampler>
  <mesh type="obj">
    <string name="filename" value="sphere.obj"/>
    <transform name="toWorld"><scale value="0.7, 0.7, 0.7"/><translate value="0, 0.7, 0"/></transform>
    <bsdf type="disney">
      <color name="baseColor" value="0.8, 0.8, 0.8"/>
      <float name="roughness" value="0.5"/>
      <string name="albedoTexture" value="tex/checker.png"/>
      <string name="normalTexture" value="tex/bumps.png"/>
      <string name="roughnessTexture" value="tex/rough.tga"/>
      <string name="specularTexture" value="tex/missing.png"/>
    </bsdf>
  </mesh>
  <mesh type="obj">
    <string name="filename" value="floor.obj"/>
    <bsdf type="diffuse">
      <color name="albedo" value="0.7 0.7 0.7"/>
      <string name="albedoTexture" value="tex/checker.png"/>
    </bsdf>
  </mesh>
  <mesh type="obj">
    <string name="filename" value="cutout.obj"/>
    <bsdf type="diffuse">
      <color name="albedo" value="0.4 0.6 0.3"/>
      <string name="alphaTexture" value="tex/leaf.bmp"/>
    </bsdf>
  </mesh>
  <mesh type="obj">
    <string name="filename" value="light.obj"/>
    <emitter type="area"><color name="radiance" value="6, 6, 6"/></emitter>
  </mesh>
</scene>
"""


@pytest.fixture(scope="module")
def tex_scene(tmp_path_factory, scenes):
    d = tmp_path_factory.mktemp("tex_scene")
    (d / "tex").mkdir()
    v, f = scenes.icosphere(3)
    v = np.asarray(v, float)
    uv = np.stack([0.5 + np.arctan2(v[:, 0], v[:, 2]) / (2 * np.pi), 0.5 + np.arcsin(np.clip(v[:, 1], -1, 1)) / np.pi], 1)
    write_obj_uv(d / "sphere.obj", v, uv, f)
    quad_f = np.array([[0, 1, 2], [0, 2, 3]])
    write_obj_uv(d / "floor.obj", np.array([[-3, 0, -3], [-3, 0, 3], [3, 0, 3], [3, 0, -3]], float),
                 np.array([[0, 0], [0, 4], [4, 4], [4, 0]], float), quad_f)
    write_obj_uv(d / "cutout.obj", np.array([[-0.6, 0.1, 1.0], [0.6, 0.1, 1.0], [0.6, 1.2, 1.0], [-0.6, 1.2, 1.0]]),
                 np.array([[0, 0], [1, 0], [1, 1], [0, 1]], float), quad_f)
    write_obj_uv(d / "light.obj", np.array([[-0.5, 3, -0.5], [0.5, 3, -0.5], [0.5, 3, 0.5], [-0.5, 3, 0.5]], float),
                 np.array([[0, 0], [1, 0], [1, 1], [0, 1]], float), quad_f)
    yy, xx = np.mgrid[0:32, 0:32]
    checker = np.where(((xx // 4) + (yy // 4)) % 2 == 0, 230, 40)[..., None].repeat(3, -1)
    checker[..., 0] = np.clip(checker[..., 0] + 20, 0, 255)
    (d / "tex" / "checker.png").write_bytes(encode_png(checker, 2, 8))
    rng = np.random.default_rng(9)
    nrm = np.stack([128 + 40 * np.sin(xx / 3.0), 128 + 40 * np.cos(yy / 4.0), np.full(xx.shape, 230)], -1)
    (d / "tex" / "bumps.png").write_bytes(encode_png(nrm.astype(np.int64), 2, 8, interlace=True))
    rough = rng.integers(20, 240, (16, 16)).astype(np.uint8)
    tga = bytes([0, 0, 3]) + bytes(9) + struct.pack("<HH", 16, 16) + bytes([8, 0x20]) + rough.tobytes()
    (d / "tex" / "rough.tga").write_bytes(tga)
    leaf = np.zeros((16, 16, 4), np.uint8)
    leaf[..., 3] = np.where((xx[:16, :16] - 8) ** 2 + (yy[:16, :16] - 8) ** 2 < 40, 255, 0)
    leaf[..., :3] = 200
    data = leaf[::-1, :, [2, 1, 0, 3]].tobytes()
    bmp = b"BM" + struct.pack("<IHHI", 54 + len(data), 0, 0, 54) + struct.pack(
        "<IiiHHIIiiII", 40, 16, 16, 1, 32, 0, len(data), 0, 0, 0, 0)
    (d / "tex" / "leaf.bmp").write_bytes(bmp + data)
    sky = np.linspace(0.2, 1.0, 16 * 8 * 3).reshape(8, 16, 3).astype(np.float32)
    write_hdr(d / "sky.hdr", sky)
    (d / "scene.xml").write_text(TEX_XML)
    return d, dict(checker=checker, nrm=nrm, rough=rough, leaf=leaf)


def scene_textures(nori, h):
    out = []
    for t in range(int(nori.nori_flat(h, 7, None))):
        info = (C.c_uint32 * 3)()
        n = nori.nori_texture(h, t, info, None)
        px = np.zeros(n, np.uint8)
        nori.nori_texture(h, t, info, px.ctypes.data)
        out.append((px.reshape(info[1], info[0], 4), bool(info[2])))
    return out


def test_scene_texture_wiring(nori, img, pt, tex_scene, capfd):
    d, src = tex_scene
    h, err = load(nori, d / "scene.xml")
    assert h, err
    mats = (pt.pt_material * 4)()
    assert nori.nori_materials(h, mats, 4) == 4
    tex = scene_textures(nori, h)
    assert "Failed to load" in capfd.readouterr().err  # tex/missing.png
    # checker (shared by two materials, one load), bumps, rough, leaf
    assert len(tex) == 4
    sph, floor, cut, light = mats
    assert floor.albedoTexIndex == sph.albedoTexIndex
    assert sph.specularTexIndex == pt.PT_NO_TEXTURE  # unreadable: the constant is used
    assert cut.alphaTexIndex != pt.PT_NO_TEXTURE and cut.albedoTexIndex == pt.PT_NO_TEXTURE
    assert light.albedoTexIndex == pt.PT_NO_TEXTURE and light.alphaTexIndex == pt.PT_NO_TEXTURE
    albedo, srgb = tex[sph.albedoTexIndex]
    assert srgb and np.array_equal(albedo[..., :3], src["checker"].astype(np.uint8)) and (albedo[..., 3] == 255).all()
    nmap, srgb = tex[sph.normalTexIndex]
    assert not srgb and np.array_equal(nmap[..., :3], src["nrm"].astype(np.uint8))
    r, srgb = tex[sph.roughnessTexIndex]
    assert not srgb and np.array_equal(r[..., 0], src["rough"])
    leaf, srgb = tex[cut.alphaTexIndex]
    assert not srgb and np.array_equal(leaf, src["leaf"])
    nori.nori_free(h)


@pytest.mark.gpu
def test_textured_xml_render_matches_direct_scene(nori, pt, tex_scene):
    """The XML path with texture maps (PNG, interlaced PNG, TGA, BMP; an alpha
    cut-out; a missing file) renders the same image as the flattened buffers
    and decoded textures uploaded through libpt directly."""
    d, _ = tex_scene
    h, err = load(nori, d / "scene.xml")
    assert h, err
    W, H = 64, 48
    s = np.zeros((H, W, 4), np.float32)
    c = np.zeros_like(s)
    st = pt.pt_stats()
    e = C.create_string_buffer(512)
    assert nori.nori_render(h, 4, 0, s.ctypes.data, c.ctypes.data, C.byref(st), e, 512) == 0, e.value
    mats = (pt.pt_material * 4)()
    nori.nori_materials(h, mats, 4)
    cam = pt.pt_camera()
    nori.nori_camera(h, C.byref(cam))
    pos, nrm, uv, tan, idx, env = (flat(nori, h, k) for k in range(6))
    ew = int(nori.nori_flat(h, 6, None))
    sc = pt.Scene(pos, idx, list(mats), normals=nrm, texcoords=uv, tangents=tan, env_rgb=env.reshape(-1, ew, 3),
                  env_scale=0.3, textures=scene_textures(nori, h))
    ctx = pt.Context(0)
    ctx.upload(sc)
    dd, _, _ = ctx.render(pt.render_params(W, H, 4, cam, max_depth=8))
    # the same scene without its maps renders differently
    plain = [pt.pt_material() for _ in range(4)]
    for k in range(4):
        C.memmove(C.byref(plain[k]), C.byref(mats[k]), C.sizeof(pt.pt_material))
        for name in ("albedoTexIndex", "normalTexIndex", "roughnessTexIndex", "alphaTexIndex"):
            setattr(plain[k], name, pt.PT_NO_TEXTURE)
    ctx.upload(pt.Scene(pos, idx, plain, normals=nrm, texcoords=uv, tangents=tan, env_rgb=env.reshape(-1, ew, 3),
                        env_scale=0.3))
    pp, _, _ = ctx.render(pt.render_params(W, H, 4, cam, max_depth=8))
    ctx.close()
    assert np.array_equal(s, dd), np.abs(s - dd).max()
    assert np.abs(pp - dd).mean() > 1e-3
    nori.nori_free(h)
