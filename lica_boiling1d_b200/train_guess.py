"""Training and evaluation of the learned initial guess (lica_unet_*).

Training data are solver problems of the pressure-Poisson workload: seeded bubble fields
(density ratio 1000, radii 8-48 cells, the bubble density of the 1024 x 1024 workload),
Gaussian right-hand sides, and the solver's operator A.  The loss is the guess's relative
residual ||f - A x0||^2 / ||f||^2 -- for a pair (f, p*) the solver produced, f = A p*, it
is the error ||A (p* - x0)||^2 / ||f||^2 in the norm the PCG's stopping test measures.  The
network works on dimensionless fields (f / rms(f), output scaled by rms(f) h^2 rho), so the
weights trained on small grids apply at any resolution.

Evaluation: PCG iterations to the same tolerance from x0 = 0 and from the guess; a guess
whose residual is not below ||f|| is replaced by zero (the fallback), so the solver alone
decides when a solution is accepted.

Usage: python -m lica_boiling1d_b200.train_guess --steps 3000 --out <weights.npy>
"""
import argparse
import os
import time

import numpy as np

from .inputs import bubble_density, face_beta

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "weights", "unet_guess.npy")


def problem(rng, n, ny=None, *, bubbles_per_1024sq=64, rmin=8.0, rmax=48.0):
    """One seeded problem of n x ny cells (h = 1/n): rho, f (zero mean), bx, by."""
    ny = n if ny is None else ny
    lam = bubbles_per_1024sq * n * ny / 1024.0 ** 2
    nb = max(1, int(rng.poisson(lam)))
    rho = bubble_density(n, ny, nbubbles=nb, rmin=rmin, rmax=rmax, seed=int(rng.integers(1 << 31)))
    f = rng.standard_normal((ny, n))
    f -= f.mean()
    bx, by = face_beta(rho)
    return rho, f, bx, by


def batch(rng, count, n):
    ps = [problem(rng, n) for _ in range(count)]
    return [np.ascontiguousarray(np.stack([p[k] for p in ps])) for k in range(4)]


def train(net, steps, n, lr=1e-3, seed=0, log_every=100, log=print, lr_final=None, anorm=True):
    """Adam steps on fresh problems of n x n (net.n per step); returns the loss history.
    anorm: the loss is the relative A-norm error against the solver's solution of each
    problem (the pair the solver generates), else the relative residual."""
    import torch
    from . import poisson
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    hist = []
    solver = poisson.MultigridPoisson(n, n, h, h, nlevels=max(2, int(np.log2(n)) - 4), ncoarse=1) if anorm else None
    t0 = time.time()
    for it in range(steps):
        lr_it = lr if lr_final is None else lr * (lr_final / lr) ** (it / max(1, steps - 1))
        rho, f, bx, by = (torch.from_numpy(a).cuda() for a in batch(rng, net.n, n))
        ps = None
        if anorm:
            ps = torch.zeros_like(f)
            for i in range(net.n):
                _, _, st = solver.solve(ps[i], f[i], bx[i], by[i], rtol=1e-10, max_iters=200)
                if st != 0:
                    raise RuntimeError(f"solver status {st} on a training problem")
        loss = net.train_step(rho, f, bx, by, h, h, lr_it, p_star=ps)
        hist.append(loss)
        if log and (it % log_every == 0 or it == steps - 1):
            log(f"step {it:5d}  loss {np.mean(hist[-log_every:]):.4e}  ({time.time() - t0:.1f} s)")
    if solver is not None:
        solver.close()
    return hist


def iterations(n, problems, guess_net=None, rtol=1e-10, nlevels=None, precision="fp64"):
    """PCG iterations (and final relative residuals) of each problem from x0 = 0, or from
    the network's guess with the zero fallback."""
    import torch
    from . import poisson
    nlevels = nlevels or max(2, int(np.log2(n)) - 4)
    s = poisson.MultigridPoisson(n, n, 1.0 / n, 1.0 / n, nlevels=nlevels, ncoarse=1, precision=precision)
    out = []
    for rho, f, bx, by in problems:
        F, BX, BY = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (f, bx, by))
        p = torch.zeros_like(F)
        if guess_net is not None:
            R = torch.from_numpy(np.ascontiguousarray(rho)).cuda()
            g, _ = guess_net.guess_checked(R[None], F[None], BX[None], BY[None], 1.0 / n, 1.0 / n)
            p.copy_(g[0])
        it, rel, st = s.solve(p, F, BX, BY, rtol=rtol, max_iters=200)
        out.append((it, rel, st))
    s.close()
    return out


def save(net, path=WEIGHTS):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.save(path, net.get_params())


def load(net, path=WEIGHTS):
    net.set_params(np.load(path))


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--n", type=int, default=256, help="training grid size")
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-final", type=float, default=1e-4)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--eval-n", type=int, default=1024)
    ap.add_argument("--eval-count", type=int, default=4)
    a = ap.parse_args()
    from .unet import LearnedGuess
    net = LearnedGuess(a.batch, a.n, a.n, seed=a.seed + 1)
    train(net, a.steps, a.n, lr=a.lr, lr_final=a.lr_final, seed=a.seed)
    save(net, a.out)
    ev = LearnedGuess(1, a.eval_n, a.eval_n)
    ev.set_params(net.get_params())
    rng = np.random.default_rng(12345)
    probs = [problem(rng, a.eval_n) for _ in range(a.eval_count)]
    base = iterations(a.eval_n, probs)
    gu = iterations(a.eval_n, probs, ev)
    print("iterations from zero :", [b[0] for b in base])
    print("iterations from guess:", [g[0] for g in gu])


if __name__ == "__main__":
    main()
