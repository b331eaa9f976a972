"""Ray hash and sort on the GPU against the reference (golden outputs of
Ref::SortRays_CPU) and the oracle: keys and permutation bit for bit."""
import numpy as np
import pytest

from raydemo_b200 import scenes
from raydemo_b200.api import Renderer

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def renderer(cuda_device):
    return Renderer(16, 16)


def gpu_sort(renderer, rays, root_min, cell, gather=True):
    import torch

    n = len(rays)
    rd = torch.from_numpy(np.ascontiguousarray(rays, np.float32)).cuda()
    keys = torch.zeros(n, dtype=torch.int32, device="cuda")
    perm = torch.zeros(n, dtype=torch.int32, device="cuda")
    out = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
    renderer.sort_rays_device(rd.data_ptr(), n, root_min, cell, perm.data_ptr(), keys.data_ptr(), out.data_ptr() if gather else 0)
    torch.cuda.synchronize()
    return keys.cpu().numpy().view(np.uint32), perm.cpu().numpy().view(np.uint32), out.cpu().numpy()


def test_golden_sort(renderer, ref_outputs):
    keys, perm, out = gpu_sort(renderer, ref_outputs["sort_rays"], ref_outputs["sort_root_min"], ref_outputs["sort_cell"])
    assert np.array_equal(keys, ref_outputs["sort_keys"])
    assert np.array_equal(perm, ref_outputs["sort_perm"])
    assert np.array_equal(out.view(np.uint32), ref_outputs["sort_rays"][perm].view(np.uint32))


@pytest.mark.parametrize("n,seed", [(1, 1), (2, 6), (255, 2), (4096, 7), (4097, 3), (3 * 8192, 8), (1 << 20, 4), (3_000_001, 5)])
def test_random_sort_vs_oracle(renderer, oracle, n, seed):
    rays = scenes.incoherent_rays(n, seed=seed)
    rays[:, 0:3] = rays[:, 0:3] * 3.0 - 1.0  # a third of the origins outside the root box on each side
    root_min = np.array([0.0, 0.0, 0.0], np.float32)
    cell = np.array([1 / 255, 1 / 255, 1 / 255], np.float32)
    keys, perm, out = gpu_sort(renderer, rays, root_min, cell)
    exp_keys = oracle.ray_hash(rays, root_min, cell)
    assert np.array_equal(keys, exp_keys)
    assert np.array_equal(perm, oracle.sort_perm(exp_keys))
    assert np.all(np.diff(keys[perm].astype(np.int64)) >= 0)
    assert np.array_equal(out.view(np.uint32), rays[perm].view(np.uint32))


def test_degenerate_grid_and_directions(renderer, oracle):
    """Zero cell size (a flat scene axis: 0/0 and x/0 in the hash), NaN and
    infinite components: the reference's x86 conversions decide the key."""
    rays = scenes.incoherent_rays(20000, seed=9)
    rays[::5, 4] = np.nan
    rays[1::5, 5] = np.inf
    rays[2::5, 0] = -np.inf
    rays[3::7, 1] = 0.0
    root_min = np.array([0.0, 0.0, 0.0], np.float32)
    cell = np.array([1 / 255, 0.0, 1 / 255], np.float32)
    keys, perm, _ = gpu_sort(renderer, rays, root_min, cell, gather=False)
    exp_keys = oracle.ray_hash(rays, root_min, cell)
    assert np.array_equal(keys, exp_keys)
    assert np.array_equal(perm, oracle.sort_perm(exp_keys))


def test_live_reference_sort(renderer, reflib):
    rays = scenes.incoherent_rays(200000, seed=10)
    rays[:, 0:3] = rays[:, 0:3] * 20.0 - 5.0
    root_min = np.array([-2.0, -1.0, 0.5], np.float32)
    cell = (np.array([12.0, 9.0, 7.0], np.float32) / np.float32(255)).astype(np.float32)
    ref_keys, ref_perm = reflib.sort_rays(rays, root_min, cell)
    keys, perm, _ = gpu_sort(renderer, rays, root_min, cell, gather=False)
    assert np.array_equal(keys, ref_keys)
    assert np.array_equal(perm, ref_perm)


@pytest.mark.parametrize("n", [5000, 300001])
def test_equal_keys_keep_input_order(renderer, oracle, n):
    """Every ray in one cell with one direction (a single digit value in
    every pass, so every tile's count sits in one digit of the look-back):
    the sort must be stable, the permutation the identity."""
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = 0.25
    rays[:, 3] = 1e30
    rays[:, 6] = 1.0
    rays[::3, 0] = 0.75  # two keys, interleaved
    root_min = np.array([0.0, 0.0, 0.0], np.float32)
    cell = np.array([1 / 255, 1 / 255, 1 / 255], np.float32)
    keys, perm, out = gpu_sort(renderer, rays, root_min, cell)
    exp_keys = oracle.ray_hash(rays, root_min, cell)
    assert np.array_equal(keys, exp_keys)
    assert np.array_equal(perm, oracle.sort_perm(exp_keys))
    assert np.array_equal(out.view(np.uint32), rays[perm].view(np.uint32))
