"""The allocation-free propagation entry point (kpax_propagate_batch_noalloc) against the
regular one (kpax_propagate_batch with an environment), through the C ABI.

The no-alloc entry exists for callers that must not allocate device memory while they run
(real-time control loops, hosts that pool all device memory); it keeps the obstacle grid in a
fixed array inside the library.  Two calls in a row with different scenes check that the shared
array is rebuilt from zero each call.  This file is named to be collected last."""
import numpy as np
import pytest

import kpax
import kpax_envs as E

pytestmark = pytest.mark.gpu
REL_TOL = 1e-5  # the propagation tolerance of the other GPU tests


def _inputs(preset, scene, seed):
    cfg = kpax.preset(preset)
    obs, _, _ = scene()
    par = E.sample_states(cfg.model, 4096, seed, cfg.v_min, cfg.v_max)
    return cfg, obs, par


def _regular(torch, cfg, obs, d_par, n, stream_id):
    d_obs = torch.from_numpy(obs).cuda()
    env = kpax.Env(cfg, d_obs.data_ptr(), obs.shape[0])
    rows = torch.zeros((n, cfg.sample_dim), device="cuda")
    valid = torch.zeros(n, dtype=torch.uint8, device="cuda")
    steps = torch.zeros(n, dtype=torch.int32, device="cuda")
    kpax.propagate_batch(cfg, env, d_par.data_ptr(), None, stream_id, n, rows.data_ptr(), valid.data_ptr(), steps.data_ptr())
    torch.cuda.synchronize()
    return rows.cpu().numpy(), valid.cpu().numpy(), steps.cpu().numpy()


def _noalloc(torch, cfg, obs, d_par, n, stream_id):
    d_obs = torch.from_numpy(obs).cuda()
    rows = torch.zeros((n, cfg.sample_dim), device="cuda")
    valid = torch.zeros(n, dtype=torch.uint8, device="cuda")
    steps = torch.zeros(n, dtype=torch.int32, device="cuda")
    kpax.propagate_batch_noalloc(cfg, d_obs.data_ptr(), obs.shape[0], d_par.data_ptr(), None, stream_id, n,
                                 rows.data_ptr(), valid.data_ptr(), steps.data_ptr())
    torch.cuda.synchronize()
    return rows.cpu().numpy(), valid.cpu().numpy(), steps.cpu().numpy()


def test_noalloc_matches_regular_entry_on_two_calls_in_a_row(cuda):
    import torch

    cases = [_inputs(kpax.PRESET_QUAD, E.quad_scene, 21), _inputs(kpax.PRESET_DI, E.di_scene, 22)]
    for call, (cfg, obs, par) in enumerate(cases):
        d_par = torch.from_numpy(par).cuda()
        n = par.shape[0]
        want_rows, want_valid, want_steps = _regular(torch, cfg, obs, d_par, n, 40 + call)
        rows, valid, steps = _noalloc(torch, cfg, obs, d_par, n, 40 + call)
        assert np.array_equal(valid, want_valid), f"call {call}: validity differs"
        assert np.array_equal(steps, want_steps), f"call {call}: executed steps differ"
        err = np.abs(rows.astype(np.float64) - want_rows) / np.maximum(np.abs(want_rows), 1.0)
        assert float(err.max()) <= REL_TOL, f"call {call}: max relative error {float(err.max())}"
        assert 0.05 < valid.mean() < 0.95


def test_noalloc_matches_phased_regular_entry_on_a_large_batch(cuda):
    """From 2^18 segments on, the regular entry runs the phased kernels (head, middle, tail with
    survivor lists in the environment's scratch) while the allocation-free entry keeps the
    one-pass kernel: both must give the same rows, verdicts and step counts."""
    import torch

    cfg = kpax.preset(kpax.PRESET_DUBINS)
    obs, _, _ = E.dubins_scene()
    n = (1 << 18) + 4099  # above the phased threshold, ragged last block
    par = E.sample_states(cfg.model, n, 23, cfg.v_min, cfg.v_max)
    d_par = torch.from_numpy(par).cuda()
    for call in range(2):
        want_rows, want_valid, want_steps = _regular(torch, cfg, obs, d_par, n, 60 + call)
        rows, valid, steps = _noalloc(torch, cfg, obs, d_par, n, 60 + call)
        assert np.array_equal(valid, want_valid), f"call {call}: validity differs"
        assert np.array_equal(steps, want_steps), f"call {call}: executed steps differ"
        err = np.abs(rows.astype(np.float64) - want_rows) / np.maximum(np.abs(want_rows), 1.0)
        assert float(err.max()) <= REL_TOL, f"call {call}: max relative error {float(err.max())}"
        assert 0.05 < valid.mean() < 0.95


def test_noalloc_rejects_inputs_beyond_its_limits(cuda):
    import torch

    cfg = kpax.preset(kpax.PRESET_DI)
    obs = E.random_boxes(5000, 3)  # more than the 4096-obstacle limit
    d_obs = torch.from_numpy(obs).cuda()
    buf = torch.zeros(64, device="cuda")
    with pytest.raises(kpax.KpaxError) as e:
        kpax.propagate_batch_noalloc(cfg, d_obs.data_ptr(), obs.shape[0], buf.data_ptr(), None, 0, 1, buf.data_ptr(),
                                     buf.data_ptr())
    assert e.value.status == kpax.ECAPACITY and "4096" in str(e.value)
    fine = kpax.preset(kpax.PRESET_DI)
    fine.hash_cell_size = 1.0  # 101^3 cells, beyond the 131072-cell limit
    with pytest.raises(kpax.KpaxError) as e:
        kpax.propagate_batch_noalloc(fine, d_obs.data_ptr(), 10, buf.data_ptr(), None, 0, 1, buf.data_ptr(), buf.data_ptr())
    assert e.value.status == kpax.ECAPACITY
