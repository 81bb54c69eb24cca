"""Export / import of built H-matrices (hm_save / hm_load through the C ABI):
the reloaded handle has the same leaves and gives bit-identical products,
densification and factorisation; factorised handles and damaged files are
refused with a status code."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(H, H2):
    assert np.array_equal(H.leaves(), H2.leaves())
    y = np.random.default_rng(7).standard_normal((H.n, 3))
    assert np.array_equal(H * y, H2 * y)
    assert np.array_equal(H.matvec(y[:, 0], trans=True), H2.matvec(y[:, 0], trans=True))


def test_save_load_aca2_roundtrip(tmp_path):
    import hmatrix as hm
    c, H = hm.NewHmat(hm.Params(Geom=np.linspace(0, 10, 4096), Kernel=hm.Cauchy(1.0), MaxBlock=512,
                                MinBlock=64, MaxRank=16, ConsMethod="aca2", εComp=1e-10, Tree="bisect",
                                Shift=1.0))
    f = tmp_path / "h.hmb"
    H.save(f)
    c2, H2 = hm.load(f)
    assert np.array_equal(c2.P, c.P) and np.array_equal(c2.X, c.X) and np.array_equal(c2.s, c.s)
    _same(H, H2)
    assert np.array_equal(H.to_dense(), H2.to_dense())
    # the reloaded handle factorises to the same L\U and solves alike
    L1, L2 = hm.lu(H), hm.lu(H2)
    assert np.array_equal(L1.to_dense(), L2.to_dense())
    b = np.random.default_rng(8).standard_normal(4096)
    assert np.array_equal(L1.solve(b), L2.solve(b))
    # a factorised handle is not saved
    with pytest.raises(hm.HmError) as e:
        L1.save(tmp_path / "lu.hmb")
    assert e.value.code == 4                                     # HM_ERR_STATE


def test_save_load_bbfmm_f32(tmp_path):
    import hmatrix as hm
    G = np.random.default_rng(2).uniform(0, 1, (2500, 2))
    c, H = hm.NewHmat(hm.Params(Geom=G, Kernel=hm.InvQuad(10.0), MaxBlock=256, MinBlock=32, MaxRank=5,
                                ConsMethod="bbfmm", Tree="bisect", Storage=hm.F32))
    f = tmp_path / "b.hmb"
    H.save(f)
    _, H2 = hm.load(f)
    _same(H, H2)
    assert H2.info().rk_entries == H.info().rk_entries


def test_damaged_files_refused(tmp_path):
    import hmatrix as hm
    _, H = hm.NewHmat(hm.Params(Geom=np.linspace(0, 1, 2048), Kernel=hm.Cauchy(1.0), MaxBlock=256,
                                MinBlock=32, MaxRank=8, ConsMethod="aca2", Tree="bisect"))
    f = tmp_path / "d.hmb"
    H.save(f)
    raw = f.read_bytes()
    (tmp_path / "cut.hmb").write_bytes(raw[: len(raw) // 2])
    (tmp_path / "junk.hmb").write_bytes(b"not an H-matrix file at all" * 8)
    (tmp_path / "tail.hmb").write_bytes(raw[:-8] + b"XXXXXXXX")
    for name in ("cut.hmb", "junk.hmb", "tail.hmb", "missing.hmb"):
        with pytest.raises(hm.HmError):
            hm.load(tmp_path / name)
    # the good file still loads after the refusals
    _, H2 = hm.load(f)
    _same(H, H2)
