"""Batch reader: MRC2014 decode (modes, byte orders, extended headers, the CTF crop), skipped
files, and batches filled with the files that load, as the reference's reader does."""
import numpy as np
import pytest
import torch

MODES = {0: np.int8, 1: np.int16, 2: np.float32, 6: np.uint16, 12: np.float16}


def write_mrc(path, data, mode=2, big_endian=False, nsymbt=0, stamp=True):
    """An MRC2014 file: 256 32-bit header words, nsymbt bytes of extended header, voxels."""
    order = ">" if big_endian else "<"
    nz, ny, nx = data.shape
    words = np.zeros(256, dtype=order + "i4")
    words[0:4] = [nx, ny, nz, mode]
    words[7:10] = [nx, ny, nz]
    words[16:19] = [1, 2, 3]
    words[23] = nsymbt
    hdr = bytearray(words.tobytes())
    hdr[52 * 4:53 * 4] = b"MAP "
    if stamp:
        hdr[212:216] = bytes([0x11, 0x11, 0, 0]) if big_endian else bytes([0x44, 0x44, 0, 0])
    else:
        hdr[212:216] = bytes(4)
    with open(path, "wb") as f:
        f.write(bytes(hdr))
        f.write(bytes(range(256)) * (nsymbt // 256) + bytes(nsymbt % 256))
        f.write(np.ascontiguousarray(data).astype(np.dtype(MODES[mode]).newbyteorder(order)).tobytes())


def _data(rng, mode, shape):
    if mode == 2:
        return rng.standard_normal(shape).astype(np.float32)
    if mode == 12:
        return (rng.standard_normal(shape) * 100).astype(np.float16)
    info = np.iinfo(MODES[mode])
    return rng.integers(info.min, info.max, shape, endpoint=True).astype(MODES[mode])


@pytest.mark.parametrize("mode", [0, 1, 2, 6, 12])
@pytest.mark.parametrize("big_endian", [False, True])
def test_decode_modes_and_byte_orders(tmp_path, mode, big_endian):
    from matcha_b200.reader import MrcReader

    rng = np.random.default_rng(mode + 10 * big_endian)
    vols = [_data(rng, mode, (12, 10, 8)) for _ in range(3)]
    paths = []
    for i, v in enumerate(vols):
        p = tmp_path / f"v{i}.mrc"
        write_mrc(p, v, mode, big_endian, nsymbt=[0, 96, 1024][i])
        paths.append(str(p))
    out, st = MrcReader(2).read(paths, (12, 10, 8))
    assert list(st) == [0, 0, 0]
    for i, v in enumerate(vols):
        np.testing.assert_array_equal(out[i].numpy(), v.astype(np.float32))


def test_decode_float16_specials_and_unstamped_files(tmp_path):
    from matcha_b200.reader import MrcReader

    v = np.array([0.0, -0.0, 1.0, -2.5, 6.0e-8, 6.1e-5, 65504.0, np.inf, -np.inf, 1e-7], np.float16)
    v = np.resize(v, (2, 3, 5)).astype(np.float16)
    write_mrc(tmp_path / "h.mrc", v, 12, stamp=False)
    write_mrc(tmp_path / "b.mrc", v.astype(np.float32), 2, big_endian=True, stamp=False)
    out, st = MrcReader(1).read([str(tmp_path / "h.mrc"), str(tmp_path / "b.mrc")], (2, 3, 5))
    assert list(st) == [0, 0]
    np.testing.assert_array_equal(out[0].numpy(), v.astype(np.float32))
    np.testing.assert_array_equal(out[1].numpy(), v.astype(np.float32))
    nan = np.full((2, 3, 5), np.nan, np.float16)
    write_mrc(tmp_path / "n.mrc", nan, 12)
    assert np.isnan(MrcReader(1).read([str(tmp_path / "n.mrc")], (2, 3, 5))[0].numpy()).all()


def test_ctf_crop(tmp_path):
    """load_ctf_relion5_cpu keeps ctf[:N//2, :, :N//2+1]."""
    from matcha_b200.reader import MrcReader, ctf_crop

    rng = np.random.default_rng(4)
    N = 16
    w = rng.random((N, N, N)).astype(np.float32)
    write_mrc(tmp_path / "w.mrc", w)
    write_mrc(tmp_path / "w1.mrc", w.astype(np.float16), 12, big_endian=True)
    out, st = MrcReader(2).read([str(tmp_path / "w.mrc"), str(tmp_path / "w1.mrc")], (N, N, N), ctf_crop(N))
    assert list(st) == [0, 0]
    np.testing.assert_array_equal(out[0].numpy(), w[:N // 2, :, :N // 2 + 1])
    np.testing.assert_array_equal(out[1].numpy(), w.astype(np.float16).astype(np.float32)[:N // 2, :, :N // 2 + 1])


def test_bad_files_report_why(tmp_path):
    from matcha_b200.reader import MrcReader

    v = np.ones((4, 4, 4), np.float32)
    write_mrc(tmp_path / "ok.mrc", v)
    write_mrc(tmp_path / "shape.mrc", np.ones((4, 4, 5), np.float32))
    write_mrc(tmp_path / "short.mrc", v)
    with open(tmp_path / "short.mrc", "r+b") as f:
        f.truncate(1024 + 100)
    (tmp_path / "junk.mrc").write_bytes(b"not an mrc file")
    write_mrc(tmp_path / "mode.mrc", v)
    with open(tmp_path / "mode.mrc", "r+b") as f:
        f.seek(12)
        f.write(np.array([4], "<i4").tobytes())  # complex64: not a subtomogram mode
    names = ["ok", "missing", "junk", "shape", "short", "mode"]
    out, st = MrcReader(3).read([str(tmp_path / f"{n}.mrc") for n in names], (4, 4, 4))
    assert list(st) == [0, 1, 2, 3, 4, 2]
    np.testing.assert_array_equal(out[0].numpy(), v)


def test_reader_rejects_bad_arguments():
    import ctypes

    from matcha_b200 import _native as nat
    from matcha_b200.reader import MrcReader

    r = MrcReader(1)
    with pytest.raises(ValueError):
        r.read_into(["x"], torch.empty((1, 4, 4, 5)), (4, 4, 4))
    st = np.zeros(1, np.int32)
    buf = torch.empty((1, 4, 4, 4))
    rc = r._lib.mtb_read_mrc(r._h, None, 1, 4, 4, 4, 4, 4, 5, buf.data_ptr(), st.ctypes.data_as(ctypes.c_void_p))
    assert rc == nat.MTB_ERR_ARG


def _dataset(tmp_path, N, n, bad=(), ctf=True):
    rng = np.random.default_rng(7)
    paths, vols, ctfs = [], [], []
    for i in range(n):
        v = rng.standard_normal((N, N, N)).astype(np.float32)
        w = rng.random((N, N, N)).astype(np.float32)
        p = tmp_path / f"TS_1/{i}_data.mrc"
        p.parent.mkdir(exist_ok=True)
        if i not in bad:
            write_mrc(p, v)
        if ctf:
            write_mrc(tmp_path / f"TS_1/{i}_weights.mrc", w)
        paths.append(str(p))
        vols.append(v)
        ctfs.append(w[:N // 2, :, :N // 2 + 1])
    return paths, vols, ctfs


def test_batches_skip_bad_files_and_fill_up(tmp_path):
    """7 files, #2 missing, batch 3: batches (0, 1, 3), (4, 5, 6) as the reference's reader
    makes them; every slot holds its files' voxels and CTF crops."""
    from matcha_b200.reader import BatchReader

    N = 8
    paths, vols, ctfs = _dataset(tmp_path, N, 7, bad=(2,))
    br = BatchReader(N, 3, do_ctf_correction=True, n_threads=2, pin=False)
    got = []
    with pytest.warns(UserWarning, match="Skipping"):
        for v, c, names, release in br.batches(paths):
            idx = [paths.index(p) for p in names]
            got.append(idx)
            for k, i in enumerate(idx):
                np.testing.assert_array_equal(v[k].numpy(), vols[i])
                np.testing.assert_array_equal(c[k].numpy(), ctfs[i])
            release()
    assert got == [[0, 1, 3], [4, 5, 6]]
    assert [p for p, _ in br.skipped] == [paths[2]]


def test_batches_without_ctf_and_a_partial_last_batch(tmp_path):
    from matcha_b200.reader import BatchReader

    N = 8
    paths, vols, _ = _dataset(tmp_path, N, 5, ctf=False)
    br = BatchReader(N, 2, do_ctf_correction=False, n_threads=1, pin=False)
    sizes = []
    for v, c, names, _release in br.batches(paths):  # no release: asking for the next batch releases
        assert c is None
        sizes.append(len(names))
        for k, p in enumerate(names):
            np.testing.assert_array_equal(v[k].numpy(), vols[paths.index(p)])
    assert sizes == [2, 2, 1]


@pytest.mark.gpu
def test_reader_feeds_align_host(tmp_path, cuda_device):
    """Batches read from MRC files and aligned through align_host give what the same
    volumes give from memory."""
    from matcha_b200.pipeline import AlignmentStep, StepConfig
    from matcha_b200.reader import BatchReader
    from tests.helpers import blob_template

    N, B = 16, 3
    rng = np.random.default_rng(31)
    tmpl = blob_template(rng, N, 12, 5, (1.0, 2.0), mask_radius=7).astype(np.float32)
    vols = (np.repeat(tmpl[None], 2 * B, 0) + 0.05 * rng.standard_normal((2 * B, N, N, N))).astype(np.float32)
    paths = []
    for i, v in enumerate(vols):
        p = tmp_path / f"{i}_data.mrc"
        write_mrc(p, v)
        paths.append(str(p))
    step = AlignmentStep(StepConfig(N=N, L=12, Li=[4, 8], batch=B, radius=7, shift_search_radius=1,
                                    shift_upsample_factor=4), cuda_device)
    step.set_template(tmpl)
    zeros3 = torch.zeros((B, 3), device=cuda_device)

    def ident():
        t = torch.zeros((B, 4), dtype=torch.float64, device=cuda_device)
        t[:, 0] = 1
        return t

    got = []
    for v, _c, names, release in BatchReader(N, B, do_ctf_correction=False).batches(paths):
        o = step.align_host(v, ident(), zeros3)
        got.append({k: o[k].clone() for k in ("alpha", "beta", "gamma", "shift")})
        release(o["copies_done"])
    torch.cuda.synchronize()
    for j in range(2):
        dv = torch.from_numpy(vols[j * B:(j + 1) * B]).to(cuda_device)
        ref = step(dv, dv, ident(), zeros3)
        for k in ("alpha", "beta", "gamma", "shift"):
            np.testing.assert_allclose(got[j][k].cpu().numpy(), ref[k].cpu().numpy(), rtol=1e-5, atol=1e-6)
