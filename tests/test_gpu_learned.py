"""Learned candidate lists: k-NN kernel, MLP gradient check, and the gain over plain k-NN."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import distances as odist
from oracle import mlp as omlp
from tsp_gpu_clean_b200 import instances

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod():
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  return torch


def test_knn_matches_distance_then_id_ranking(torch_mod):
  from oracle import distances as odist
  from tsp_gpu_clean_b200 import learned

  coords = instances.clustered_instance(700, 5, 20.0, 3)
  coords[10:20] = coords[0]  # coincident points: many distance ties
  inst = learned.device_instance(coords, 30)
  got = inst.pool.cpu().numpy()
  D = odist.euc2d_matrix(coords).astype(np.int64)
  n = len(coords)
  np.fill_diagonal(D, np.iinfo(np.int64).max)
  ids = np.broadcast_to(np.arange(n), (n, n))
  want = np.stack([np.lexsort((ids[u], D[u]))[:30] for u in range(n)])
  assert np.array_equal(got, want)
  inst2 = learned.device_instance(coords, 30, with_matrix=False)  # rebuilt FP64 distances
  assert np.array_equal(inst2.pool.cpu().numpy(), want)


def test_mlp_forward_gradients_and_adam_match_oracle(torch_mod):
  torch = torch_mod
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle
  from tsp_gpu_clean_b200.learned import EdgeScorer

  rng = np.random.default_rng(7)
  E = 3001
  feats = rng.uniform(-2, 2, (E, 5)).astype(np.float32)
  x = np.zeros((E, 16), dtype=np.float32)
  x[:, :5] = feats
  y = (rng.random(E) < 0.2).astype(np.float32)
  sc = EdgeScorer(seed=3)
  p = sc.params.cpu().numpy()
  p[omlp.O_B1 : omlp.O_W2] = rng.normal(0, 0.1, 64)
  p[omlp.O_B2 : omlp.O_W3] = rng.normal(0, 0.1, 64)
  sc.params.copy_(torch.from_numpy(p))
  xb16 = (omlp.bf16(x).view(np.uint32) >> 16).astype(np.uint16).view(np.int16)
  dx = torch.from_numpy(xb16.copy()).cuda()
  logits = sc.logits(dx).cpu().numpy()
  _, _, _, want = omlp.forward(p, x)
  np.testing.assert_allclose(logits, want, rtol=2e-3, atol=2e-3)
  loss = torch.zeros(1, dtype=torch.float32, device="cuda")
  grad = torch.zeros_like(sc.params)
  dy = torch.from_numpy(y).cuda()
  native.call("tspb_mlp_train_grad", ptr(sc.params), ptr(dx), ptr(dy), E, ptr(grad), ptr(loss), stream_handle())
  g_want, l_want = omlp.grads(p, x, y)
  g = grad.cpu().numpy()
  scale = np.abs(g_want).max()
  np.testing.assert_allclose(g, g_want, rtol=0, atol=3e-3 * scale)
  assert abs(float(loss.item()) - l_want) <= 1e-3 * abs(l_want)
  # one Adam step on the GPU gradient, compared with the oracle's update of the same gradient
  m = np.zeros_like(p)
  v = np.zeros_like(p)
  p_want, _, _ = omlp.adam(p, g, m, v, 1)
  sc.grad.copy_(grad)
  native.call("tspb_mlp_adam", ptr(sc.params), ptr(sc.grad), ptr(sc.m), ptr(sc.v), 1, 3e-3, 0.9, 0.999, 1e-8, 0.0,
              stream_handle())
  np.testing.assert_allclose(sc.params.cpu().numpy(), p_want, rtol=1e-5, atol=1e-6)


def test_learned_candidates_beat_plain_knn_at_equal_size(torch_mod):
  """Trained on good tours of 48 generated instances, the learned top-8 lists hold more
  of a held-out instance's good-tour edges than the 8 nearest neighbours, and 2-opt with
  them reaches shorter tours from the same starts."""
  from tsp_gpu_clean_b200 import learned

  lc = learned.LearnedCandidates(pool_k=24, seed=0)
  rng = np.random.default_rng(11)
  xs, ys = [], []
  for i in range(48):
    n = int(rng.integers(200, 600))
    coords = instances.uniform_instance(n, 1000 + i) if i % 2 else instances.clustered_instance(n, int(rng.integers(5, 20)), 40.0, 1000 + i)
    inst = learned.device_instance(coords, 24)
    tour = lc.label_tour(inst, starts=4, seed=i)
    x, y = lc.training_edges(inst, tour)
    xs.append(x)
    ys.append(y)
  lc.fit(xs, ys, epochs=4, batch=1 << 14, lr=3e-3)
  assert np.mean(lc.train_log[-10:]) < np.mean(lc.train_log[:10])
  rec_l, rec_k, len_l, len_k = [], [], [], []
  for j in range(6):
    coords = instances.uniform_instance(500, 5000 + j) if j % 2 else instances.clustered_instance(500, 12, 40.0, 5000 + j)
    inst = learned.device_instance(coords, 24)
    good = lc.label_tour(inst, starts=8, seed=100 + j)
    tab_l = lc.table(inst, 8)
    tab_k = inst.pool[:, :8].contiguous()
    rec_l.append(learned.edge_recall(tab_l, good))
    rec_k.append(learned.edge_recall(tab_k, good))
    starts = learned.random_starts(500, 16, 200 + j)
    t_l, _ = learned.two_opt_table(inst, starts, tab_l, mode="best")
    t_k, _ = learned.two_opt_table(inst, starts, tab_k, mode="best")
    len_l.append(learned.tour_lengths(inst, t_l).mean())
    len_k.append(learned.tour_lengths(inst, t_k).mean())
  print("recall learned/knn", np.mean(rec_l), np.mean(rec_k), "2-opt length learned/knn", np.mean(len_l), np.mean(len_k))
  assert np.mean(rec_l) > np.mean(rec_k)
  assert np.mean(len_l) < np.mean(len_k)


def test_iterated_two_opt_under_a_budget():
  """Double-bridge kicks keep permutations; iterated 2-opt never ends above its first
  descent and stops once the CUDA-event budget is used."""
  import torch

  if not torch.cuda.is_available():
    pytest.skip("no CUDA device")
  from tsp_gpu_clean_b200 import learned
  from tsp_gpu_clean_b200.build import build_library

  build_library()
  coords = instances.uniform_instance(400, 77)
  inst = learned.device_instance(coords, 30)
  g = torch.Generator().manual_seed(3)
  base = torch.randperm(400, generator=g).to(torch.int32).cuda()
  kicked = learned.double_bridge(base, 16, g)
  assert kicked.shape == (16, 400)
  for row in kicked.cpu().numpy():
    assert np.array_equal(np.sort(row), np.arange(400))
  starts = learned.nn_starts(inst, 4, 5)
  table = inst.pool[:, :10].contiguous()
  first, _ = learned.two_opt_table(inst, starts, table, mode="best")
  first_best = float(learned.tour_lengths(inst, first).min())
  res = learned.iterated_two_opt(inst, starts, table, budget_s=0.05, kicks=32, seed=1)
  assert res["length"] <= first_best and res["rounds"] >= 1 and res["used_s"] >= 0.05
  t = res["tour"].cpu().numpy()
  assert np.array_equal(np.sort(t), np.arange(400))
  D = odist.euc2d_matrix(coords)
  assert int(D[t, np.roll(t, -1)].sum()) == int(res["length"])


@pytest.mark.parametrize("E", [128, 3001, 70000])
def test_tensor_core_gradient_matches_oracle_and_mma_sync_kernel(torch_mod, E):
  """The tcgen05 training gradient (tensor-memory accumulators, 128-edge tiles, partial last
  tile) against the NumPy oracle with its rounding points (dh1 in BF16 for dW1/db1) and
  against the mma.sync kernel, within the tolerances of the oracle test above."""
  torch = torch_mod
  from tsp_gpu_clean_b200 import native
  from tsp_gpu_clean_b200.device import ptr, stream_handle
  from tsp_gpu_clean_b200.learned import EdgeScorer

  rng = np.random.default_rng(11 + E)
  feats = rng.uniform(-2, 2, (E, 5)).astype(np.float32)
  x = np.zeros((E, 16), dtype=np.float32)
  x[:, :5] = feats
  y = (rng.random(E) < 0.2).astype(np.float32)
  sc = EdgeScorer(seed=5)
  p = sc.params.cpu().numpy()
  p[omlp.O_B1 : omlp.O_W2] = rng.normal(0, 0.1, 64)
  p[omlp.O_B2 : omlp.O_W3] = rng.normal(0, 0.1, 64)
  sc.params.copy_(torch.from_numpy(p))
  xb16 = (omlp.bf16(x).view(np.uint32) >> 16).astype(np.uint16).view(np.int16)
  dx = torch.from_numpy(xb16.copy()).cuda()
  dy = torch.from_numpy(y).cuda()
  out = {}
  for name in ("tspb_mlp_train_grad_tc", "tspb_mlp_train_grad"):
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    grad = torch.zeros_like(sc.params)
    if name.endswith("_tc"):
      status = torch.zeros(1, dtype=torch.int32, device="cuda")
      native.call(name, ptr(sc.params), ptr(dx), ptr(dy), E, ptr(grad), ptr(loss), ptr(status), stream_handle())
      assert int(status.item()) == 0
    else:
      native.call(name, ptr(sc.params), ptr(dx), ptr(dy), E, ptr(grad), ptr(loss), stream_handle())
    out[name] = (grad.cpu().numpy(), float(loss.item()))
  g_tc, l_tc = out["tspb_mlp_train_grad_tc"]
  g_mma, _ = out["tspb_mlp_train_grad"]
  g_want, l_want = omlp.grads(p, x, y, dh1_bf16=True)
  scale = np.abs(g_want).max()
  np.testing.assert_allclose(g_tc, g_want, rtol=0, atol=3e-3 * scale)
  np.testing.assert_allclose(g_tc, g_mma, rtol=0, atol=3e-3 * scale)
  assert abs(l_tc - l_want) <= 1e-3 * abs(l_want)
