"""Host-side file formats: FITS cubes (MATLAB fitswrite layout) and MATLAB
v5 checkpoints under the reference's field names.  No GPU."""
import numpy as np

from fhs_b200 import io


def test_fits_round_trip_and_layout(tmp_path):
    x = np.random.default_rng(0).standard_normal((6, 5, 3))
    p = tmp_path / "cube.fits"
    io.fitswrite(x, p)
    raw = p.read_bytes()
    assert len(raw) % 2880 == 0
    assert raw[:80] == b"SIMPLE  =                    T / conforms to FITS standard".ljust(80)
    assert raw[80:160] == b"BITPIX  =                  -64".ljust(80)
    assert raw[160:240] == b"NAXIS   =                    3".ljust(80)
    assert raw[240:320] == b"NAXIS1  =                    6".ljust(80)
    # data: big-endian doubles, NAXIS1 (MATLAB rows) fastest
    d = np.frombuffer(raw, dtype=">f8", count=x.size, offset=2880)
    assert np.array_equal(d, x.reshape(-1, order="F"))
    y, hdr = io.fitsread(p, with_header=True)
    assert hdr["NAXIS"] == 3 and (hdr["NAXIS1"], hdr["NAXIS2"], hdr["NAXIS3"]) == (6, 5, 3)
    assert y.shape == x.shape and np.array_equal(y, x)


def test_fits_float32_and_scaled_integers(tmp_path):
    x = np.linspace(-1, 1, 24).reshape(4, 6)
    p = tmp_path / "img.fits"
    io.fitswrite(x, p, bitpix=-32, header=[("object", "test")])
    y, hdr = io.fitsread(p, with_header=True)
    assert hdr["OBJECT"] == "test" and hdr["BITPIX"] == -32
    assert np.array_equal(y, x.astype(np.float32).astype(np.float64))
    # a 16-bit image with BSCALE / BZERO written by hand
    cards = [b"SIMPLE  =                    T", b"BITPIX  =                   16", b"NAXIS   =                    1",
             b"NAXIS1  =                    3", b"BSCALE  =                  0.5", b"BZERO   =                 10.0",
             b"END"]
    head = b"".join(c.ljust(80) for c in cards)
    head += b" " * (-len(head) % 2880)
    data = np.array([0, 2, -4], dtype=">i2").tobytes()
    (tmp_path / "s.fits").write_bytes(head + data + b"\0" * (2880 - len(data)))
    assert np.array_equal(io.fitsread(tmp_path / "s.fits"), [10.0, 11.0, 8.0])


def test_checkpoint_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    state = {
        "xsol": rng.random((8, 6, 4)),
        "g": rng.standard_normal((8, 6, 4)),
        "v0": rng.standard_normal(50),
        "v1": rng.standard_normal((30, 4)),
        "v2": [[rng.standard_normal(5) + 1j * rng.standard_normal(5), rng.standard_normal(3) + 0j]
               for _ in range(4)],
        "weights0": rng.random((4, 2, 2)),
        "weights1": rng.random((30, 2)),
        "epsilon": [[1.5, 2.25] for _ in range(4)],
    }
    p = tmp_path / "ckpt.mat"
    io.save_checkpoint(p, state, end_iter=17, rel_val=np.array([0.1, 0.01]))
    back = io.load_checkpoint(p)
    for k in ("xsol", "g", "v1", "weights0", "weights1"):
        assert np.array_equal(back[k], state[k]), k
    assert np.array_equal(back["v0"], state["v0"])
    for l in range(4):
        for b in range(2):
            assert np.array_equal(back["v2"][l][b], state["v2"][l][b])
    assert back["epsilon"] == state["epsilon"]
    assert int(back["end_iter"].ravel()[0]) == 17


def test_channel_data_file_conversion(tmp_path):
    """u, v in wavelengths -> radians at the given pixel size; y and G rows
    weighted by nW .* nWimag (the reference's data whitening)."""
    from scipy.io import savemat
    rng = np.random.default_rng(5)
    n = 40
    u, v, w = rng.uniform(-1e3, 1e3, (3, n))
    nW, nWimag = rng.uniform(0.5, 2.0, (2, n))
    y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    savemat(tmp_path / "ch1.mat", dict(u=u[:, None], v=v[:, None], w=w[:, None], nW=nW[:, None],
                                       nWimag=nWimag[:, None], y=y[:, None], frequency=1.4e9,
                                       maxProjBaseline=1.5e3))
    px = io.nominal_pixel_size(1.5e3, 2.0)
    d = io.load_channel_data(tmp_path / "ch1.mat", px)
    hsb = (180 / np.pi) * 3600 / px / 2
    assert np.allclose(d["om_x"], u * np.pi / hsb) and np.allclose(d["om_y"], -v * np.pi / hsb)
    # at the nominal 2x super-resolution the longest baseline maps to pi/2
    assert np.isclose(np.pi * 1.5e3 / hsb, np.pi / 2)
    assert np.allclose(d["weights"], nW * nWimag) and np.allclose(d["y"], y * nW * nWimag)
    assert d["frequency"] == 1.4e9 and d["max_proj_baseline"] == 1.5e3
    d2 = io.load_channel_data(tmp_path / "ch1.mat", px, apply_imaging_weights=False)
    assert np.allclose(d2["weights"], nW)


def test_update_epsilon_rule():
    """src/update_epsilon.m:52-71: blocks outside [tol_in, tol_out] x eps move
    towards the residual, at most once per adapt_eps_steps iterations."""
    from fhs_b200.heuristics import update_epsilon
    eps, tb = update_epsilon([[10.0, 10.0, 10.0]], 50, [[0, 0, 45]], [[5.0, 20.0, 5.0]], 0.99, 1.001, 10, 0.5)
    assert eps == [[7.5, 15.0, 10.0]] and tb == [[50, 50, 45]]
    eps, tb = update_epsilon([[10.0]], 50, [[0]], [[10.0]], 0.99, 1.001, 10, 0.5)
    assert eps == [[10.0]] and tb == [[0]]
