"""The bench's full-size parity check (bench.parity_vs_reference) on a small
synthetic fixture in the committed fixture's format: per-chunk digests of the
reference's (prim, t, u, v) records, the rays where the reference's answer
deviates from the order-independent closest hit (with the answer this tracer
gives there and the reference's), and the hit count. Equal records pass;
a listed deviation where this tracer gives its closest hit is mapped and
counted as explained; any other difference shows as a mismatching chunk."""
import numpy as np

import bench


def _fixture(path, tris, rays, ref, dev_idx, dev_ours, dev_kind, chunk=4):
    np.savez(path, chunk=np.int64(chunk), mb_inputs_sha256=np.bytes_(bench.inputs_sha256(tris, rays)),
             mb_digests=bench.chunk_digests(ref, chunk), mb_hits=np.int64(np.sum(ref[:, 0].view(np.int32) >= 0)),
             mb_dev_idx=np.asarray(dev_idx, np.int64), mb_dev_ours=np.asarray(dev_ours, np.uint32).reshape(-1, 4),
             mb_dev_ref=ref[np.asarray(dev_idx, np.int64)].reshape(-1, 4), mb_dev_kind=np.asarray(dev_kind, np.int64))


def _case(n=22, seed=5):
    rng = np.random.default_rng(seed)
    tris = rng.random((6, 3, 3)).astype(np.float32)
    rays = rng.random((n, 8)).astype(np.float32)
    ref = rng.integers(0, 1 << 30, (n, 4)).astype(np.uint32)
    ref[::5, 0] = np.uint32(0xFFFFFFFF)  # misses
    return tris, rays, ref


def test_equal_records_pass(tmp_path):
    tris, rays, ref = _case()
    fx = str(tmp_path / "fx.npz")
    _fixture(fx, tris, rays, ref, [], [], [])
    out = bench.parity_vs_reference("mb", tris, rays, ref.copy(), fixture=fx)
    assert out["mismatch"] == 0 and out["unexplained_deviation_rays"] == 0
    assert out["hits"] == out["ref_hits"] == int(np.sum(ref[:, 0].view(np.int32) >= 0))


def test_listed_deviation_is_explained_and_others_are_not(tmp_path):
    tris, rays, ref = _case()
    ours = ref.copy()
    ours[7] = (3, 111, 222, 333)  # the reference kept another triangle at the same t: a listed tie
    fx = str(tmp_path / "fx.npz")
    _fixture(fx, tris, rays, ref, [7], [ours[7]], [0])
    out = bench.parity_vs_reference("mb", tris, rays, ours, fixture=fx)
    assert out["mismatch"] == 0 and out["explained"]["exact_t_ties"] == 1
    other = ours.copy()
    other[13, 1] ^= 1  # one bit of t elsewhere
    out = bench.parity_vs_reference("mb", tris, rays, other, fixture=fx)
    assert out["mismatch_chunks"] == 1 and out["bad_chunks"] == [13 // 4]
    wrong = ours.copy()
    wrong[7] = (4, 111, 222, 333)  # at the listed ray, neither answer
    out = bench.parity_vs_reference("mb", tris, rays, wrong, fixture=fx)
    assert out["unexplained_deviation_rays"] == 1 and out["mismatch_chunks"] == 1


def test_other_inputs_are_not_compared(tmp_path):
    tris, rays, ref = _case()
    fx = str(tmp_path / "fx.npz")
    _fixture(fx, tris, rays, ref, [], [], [])
    rays2 = rays.copy()
    rays2[0, 0] += 1.0
    out = bench.parity_vs_reference("mb", tris, rays2, ref, fixture=fx)
    assert out["mismatch"] is None and "differ" in out["fixture"]
    assert bench.parity_vs_reference("mb", tris, rays, ref, fixture=str(tmp_path / "absent.npz"))["fixture"] == "absent"
