"""Headless viewer images (grn_render_cells / grn_render_concentrations /
grn_write_ppm) against a numpy restatement of the reference viewer's image
threads."""
import numpy as np

import grn_b200 as grn

PALETTE = [0xFF0000, 0x00FF00, 0x0000FF, 0xFF00FF, 0xFFFF00, 0x00FFFF, 0xC0C0C0, 0x7425B1,
           0xFF9233, 0xAD2323, 0xFED4D9, 0x5F6142, 0x43B3AE, 0xFEDA83, 0x814A19, 0xC0D8F2,
           0xC3C982, 0xE88F2B, 0x868A35]


def _planes(rng, n, H, W):
    p = rng.uniform(-0.2, 1.6, size=(n, H, W)).astype(np.float32)
    p[0, 0, 0] = np.nan
    p[-1, -1, -1] = 1.0
    return p


def _cells_ref(p, n_morph):
    out = np.zeros(p.shape[1:] + (3,), np.uint8)
    for k in range(n_morph):
        c = p[k].astype(np.float64)
        v = 255.0 * np.where(c < 1.0, c, 1.0)
        v = np.where(np.isnan(v), 0, v)
        out[..., k] = (np.trunc(v).astype(np.int64) & 0xff).astype(np.uint8)
    return out


def _conc_ref(p, factor):
    H, W = p.shape[1:]
    out = np.zeros((H, W, 3), np.uint8)
    for y in range(H):
        for x in range(W):
            acc = [0, 0, 0]
            for k in range(p.shape[0]):
                f = float(p[k, y, x]) / factor
                c = PALETTE[k % 19]
                for ch, sh in enumerate((16, 8, 0)):
                    v = acc[ch] + ((c >> sh) & 0xff) * f
                    acc[ch] = acc[ch] if np.isnan(v) else int(v)  # C++ truncation
            out[y, x] = [min(a, 255) & 0xff for a in acc]
    return out


def test_render_cells(built_libs):
    rng = np.random.default_rng(0)
    p = _planes(rng, 4, 7, 9)
    for n_morph in (1, 2, 3):
        np.testing.assert_array_equal(grn.render_cells(p, n_morph), _cells_ref(p, n_morph))


def test_render_concentrations(built_libs):
    rng = np.random.default_rng(1)
    p = _planes(rng, 21, 5, 6)  # > 19 products: the palette wraps
    for factor in (1.0, 0.5, 3.0):
        np.testing.assert_array_equal(grn.render_concentrations(p, factor), _conc_ref(p, factor))


def test_write_ppm(built_libs, tmp_path):
    rgb = np.random.default_rng(2).integers(0, 256, size=(5, 7, 3), dtype=np.uint8)
    path = tmp_path / "frame.ppm"
    grn.write_ppm(path, rgb)
    data = path.read_bytes()
    header = b"P6\n7 5\n255\n"
    assert data.startswith(header)
    np.testing.assert_array_equal(np.frombuffer(data[len(header):], np.uint8).reshape(5, 7, 3),
                                  rgb)
