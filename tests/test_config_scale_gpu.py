"""Parity at the stated configuration sizes (the other GPU tests use reduced sizes):

* the 64-lattice batch of D2Q9 MRT cavities in fp16 (edges log-uniform in [128, 1024],
  tau ~ U[0.51, 1], U ~ U[0.05, 0.1]) after the full 2000 steps: every lattice's velocity
  field against the float64 oracle run on the device. The error is that of fp16 storage
  itself: on the worst lattices and the tau-minimum one it is within 1.5x the error of the
  float64 oracle whose state is rounded to fp16 (f - w) after every step, and every lattice
  stays within 2e-2 U (measured: 1.05e-2 U at worst, near the lid corners of the largest
  cavity; median 4e-3 U);
* the 1024 x 256 adjoint channel (disc of diameter 40 at (200, 129), tau 0.56, g_x = 1e-6,
  control field N(0, 1e-7), T = 2000, t0 = 1500, checkpoints every 45 steps): J agrees with
  the float64 oracle's J, the gradient is finite and zero on solid nodes; on a cropped time
  window (T = 40, t0 = 30) the full gradient equals torch autograd through the float64
  oracle at full size within 1e-4, also along random directions.

The float64 oracle runs as torch float64 tensors on the GPU; each oracle step is captured
once in a CUDA graph and replayed, several lattices on separate streams.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import lbm_oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _oracle_graph_runs(cases: list, f0s: list, steps: int, streams: int = 8) -> list:
    """float64 oracle states after ``steps`` steps for each (case, f0), every step replayed
    from a CUDA graph of one oracle step, ``streams`` lattices at a time. Every tensor a
    captured graph reads or writes stays referenced until the graph is released."""
    out = [None] * len(cases)
    order = sorted(range(len(cases)), key=lambda i: -f0s[i].numel())
    for start in range(0, len(order), streams):
        chunk = order[start:start + streams]
        work = []
        for i in chunk:
            st = torch.cuda.Stream()
            st.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(st):
                fin = f0s[i].clone()
                O.step(fin, cases[i], torch)  # lazy initialisation outside the capture
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=st):
                    fin.copy_(O.step(fin, cases[i], torch))
            work.append((i, st, g, fin))
        for _ in range(steps):
            for _, st, g, _ in work:
                with torch.cuda.stream(st):
                    g.replay()
        for i, st, g, fin in work:
            torch.cuda.current_stream().wait_stream(st)
            out[i] = fin.clone()
        torch.cuda.synchronize()
        del work
    return out


def _oracle_f16_storage_run(case, f0, steps: int):  # noqa: ANN001, ANN202
    """The float64 oracle with its state rounded as fp16 storage of f - w after every step
    (plain launches, no graph)."""
    w = torch.as_tensor(case.lat.w, dtype=torch.float64, device="cuda")
    w = w.view((-1,) + (1,) * case.dim)
    f = f0.clone()
    for _ in range(steps):
        f = (O.step(f, case, torch) - w).to(torch.float16).to(torch.float64) + w
    return f


def test_config4_full_batch_velocity_against_float64():
    from pylbm_b200 import workloads as W
    from pylbm_b200.batched import BatchedSolver

    probs = W.cavity_batch_problems(64, seed=0, collision="mrt")
    assert len(probs) == 64 and max(max(p.shape) for p in probs) > 900
    b = BatchedSolver(probs, "fused-fp16")
    b.step(2000)
    vel = [b.velocity(i).double() for i in range(len(probs))]
    b.close()
    cases = [O.Case.from_problem(p) for p in probs]
    f0s = [torch.as_tensor(p.initial_populations(), device="cuda") for p in probs]
    refs = _oracle_graph_runs(cases, f0s, 2000)
    u_refs = [torch.stack(list(O.macroscopic(refs[i], cases[i])[1])) for i in range(64)]
    errs = [float((vel[i] - u_refs[i]).abs().max().item()) / p.u_lid
            for i, p in enumerate(probs)]
    worst = int(np.argmax(errs))
    print(f"\nconfig4 fp16 MRT, 64 lattices x 2000 steps: velocity L-inf / U max {max(errs):.3e} "
          f"(lattice {worst}: {probs[worst].shape}, tau {probs[worst].tau:.4f}, "
          f"U {probs[worst].u_lid:.4f}), median {np.median(errs):.3e}")
    tmin = min(range(64), key=lambda i: probs[i].tau)
    print(f"  tau-min lattice {tmin} (tau {probs[tmin].tau:.4f}): {errs[tmin]:.3e}")
    assert all(np.isfinite(errs))
    assert max(errs) <= 2e-2, errs
    # the same lattices with fp16 storage rounding emulated in the float64 oracle
    check = sorted(set(np.argsort(errs)[-3:].tolist() + [tmin]))
    for i in check:
        emul = _oracle_f16_storage_run(cases[i], f0s[i], 2000)
        u_e = torch.stack(list(O.macroscopic(emul, cases[i])[1]))
        e_emul = float((u_e - u_refs[i]).abs().max().item()) / probs[i].u_lid
        print(f"  lattice {i}: kernel {errs[i]:.3e} U, fp16-rounded float64 {e_emul:.3e} U")
        assert errs[i] <= 1.5 * e_emul + 1e-4, (i, errs[i], e_emul)


def _channel_problem():
    from pylbm_b200 import workloads as W
    from pylbm_b200.problem import Problem

    solid, F = W.cylinder_channel(1024, 256, 200.0, 129.0, 40.0, 1e-7, seed=0)
    p = Problem((1024, 256), tau=0.56, periodic=(True, False), force=(1e-6, 0.0), solid=solid)
    return p, solid, F


def _oracle_case(p, solid, field):  # noqa: ANN001, ANN202
    return O.Case(p.shape, p.tau, "bgk", p.periodic, 0.0, p.force, solid=solid,
                  force_field=field)


def test_config5_full_size_objective_and_gradient():
    from pylbm_b200.adjoint import DragAdjoint

    p, solid, F = _channel_problem()
    adj = DragAdjoint(p, steps=2000, t0=1500, checkpoint=45)
    Fd = torch.as_tensor(F, dtype=torch.float32, device="cuda")
    J = adj.objective(Fd)
    g = adj.gradient()
    assert np.isfinite(J) and bool(torch.isfinite(g).all())
    assert float(g.abs().max().item()) > 0.0
    assert float(g[:, torch.as_tensor(solid, device="cuda")].abs().max().item()) == 0.0
    assert len(adj._checkpoints) == 45  # ceil(2000 / 45)
    # J of the float64 oracle (fp32 control field as float64), plain forward on the device
    case = _oracle_case(p, solid, torch.as_tensor(F.astype(np.float32).astype(np.float64),
                                                  device="cuda"))
    f0 = torch.as_tensor(p.initial_populations(), device="cuda")
    with torch.no_grad():
        J64 = float(O.drag_objective(case, f0, 2000, 1500, xp=torch))
    print(f"\nconfig5 1024x256: J = {J:.9e} (float64 oracle {J64:.9e}), "
          f"max|dJ/dF| = {float(g.abs().max().item()):.3e}")
    assert J == pytest.approx(J64, rel=1e-4)


def test_config5_full_size_gradient_matches_autograd_on_a_window():
    from pylbm_b200.adjoint import DragAdjoint

    p, solid, F = _channel_problem()
    T, t0 = 40, 30
    adj = DragAdjoint(p, steps=T, t0=t0, checkpoint=15)
    F32 = F.astype(np.float32)
    adj.objective(torch.as_tensor(F32, device="cuda"))
    grad = adj.gradient()
    Ft = torch.tensor(F32.astype(np.float64), device="cuda", requires_grad=True)
    case = _oracle_case(p, solid, Ft)
    J = O.drag_objective(case, torch.as_tensor(p.initial_populations(), device="cuda"), T, t0,
                         xp=torch, checkpoint=10)
    J.backward()
    ref = Ft.grad
    rel = float(torch.linalg.norm(grad - ref) / torch.linalg.norm(ref))
    print(f"\nconfig5 window T={T}: |dJ/dF - autograd| / |autograd| = {rel:.3e}")
    assert rel < 1e-4
    gen = torch.Generator(device="cuda").manual_seed(7)
    fluid = torch.as_tensor(~solid, device="cuda", dtype=torch.float64)
    for _ in range(3):
        v = torch.randn(ref.shape, generator=gen, device="cuda", dtype=torch.float64) * fluid
        a, r = float((grad * v).sum()), float((ref * v).sum())
        assert a == pytest.approx(r, rel=1e-4)
