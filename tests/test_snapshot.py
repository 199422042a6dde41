"""Checkpoint files (checkpoint.f90 / particle_initialization.f90 format) written and read
through the C ABI; host code, no GPU."""
import struct

import numpy as np
import pytest


def _image():
    from cube2_b200.layout import Layout, build_image
    L = Layout(ng=32, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1)
    rng = np.random.default_rng(21)
    pos = rng.random((3000, 3)) * 32
    vel = rng.standard_normal((3000, 3)).astype(np.float32)
    return L, build_image(pos, vel, L)


def test_file_names_follow_the_reference():
    from cube2_b200.snapshot import file_names
    assert file_names("/out/", 1, 0.0) == ("/out/image1/0.000_", "_1.bin")
    assert file_names("/out/", 12, 10.5) == ("/out/image12/10.500_", "_12.bin")


def test_written_files_have_the_reference_layout(tmp_path):
    from cube2_b200 import snapshot as S
    L, img = _image()
    prefix, suffix = S.file_names(str(tmp_path) + "/", 1, 0.0)
    (tmp_path / "image1").mkdir()
    h = S.default_header(L)
    h.update(timestep=7, a=0.5, box=100.0, sigma_vi=0.25, vz_max=1.5)
    S.write(img, prefix, suffix, h)
    n = int(img.active.sum())
    info = open(prefix + "info" + suffix, "rb").read()
    assert len(info) == S.HEADER_BYTES == 180
    ints = struct.unpack("<13q", info[:104])
    reals = struct.unpack("<19f", info[104:])
    assert ints[0] == n and ints[1] == img.n_particles and ints[2:4] == (2, 2) and ints[10] == 7
    assert ints[6:8] == (L.nnt, L.nt)
    assert reals[0] == 0.5 and reals[9] == 100.0 and reals[16] == 0.25 and reals[18] == 1.5
    xp = np.fromfile(prefix + "xp" + suffix, np.int16).reshape(-1, 3)
    vp = np.fromfile(prefix + "vp" + suffix, np.float32).reshape(-1, 3)
    pid = np.fromfile(prefix + "id" + suffix, np.int64)
    npc = np.fromfile(prefix + "np" + suffix, np.int32)
    # the physical copies in storage order: tile by tile, row by row, cell by cell
    np.testing.assert_array_equal(xp, img.xp[img.active])
    np.testing.assert_array_equal(vp, img.vp[img.active])
    np.testing.assert_array_equal(pid, img.pid[img.active])
    nt, ncb = L.nt, L.ncb
    np.testing.assert_array_equal(npc, img.rhoc[:, :, :, ncb:ncb + nt, ncb:ncb + nt, ncb:ncb + nt].reshape(-1))
    # and read back
    h2, phys, x2, v2, p2 = S.read_physical(L, prefix, suffix)
    assert h2["nplocal"] == n and h2["timestep"] == 7 and h2["a"] == 0.5
    np.testing.assert_array_equal(x2, xp)
    np.testing.assert_array_equal(v2, vp)
    np.testing.assert_array_equal(p2, pid)
    np.testing.assert_array_equal(phys.reshape(-1), npc)


def test_read_rejects_other_formats_and_small_capacity(tmp_path):
    import ctypes
    from cube2_b200 import snapshot as S
    from cube2_b200.kick import lib
    L, img = _image()
    prefix, suffix = str(tmp_path) + "/a_", "_1.bin"
    S.write(img, prefix, suffix)
    c = S.CSimHeader()
    xp = np.zeros((10, 3), np.int16)
    vp = np.zeros((10, 3), np.float32)
    rc = lib().cube_snapshot_read(prefix.encode(), suffix.encode(), ctypes.byref(c), None,
                                  xp.ctypes.data_as(ctypes.c_void_p), vp.ctypes.data_as(ctypes.c_void_p), None,
                                  ctypes.c_int64(10))
    assert rc == 5 and c.nplocal == int(img.active.sum())
    h = S.default_header(L)
    h["izipx"] = 4  # another stored format: refused as the reference does
    S.write(img, prefix, suffix, h)
    rc = lib().cube_snapshot_read(prefix.encode(), suffix.encode(), ctypes.byref(c), None, None, None, None,
                                  ctypes.c_int64(0))
    assert rc == 1
    with pytest.raises(Exception):
        S.read_physical(L, str(tmp_path) + "/missing_", suffix)
