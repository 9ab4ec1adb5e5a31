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
FILM_WEIGHTS = os.path.join(HERE, "weights", "unet_guess_film.npy")
# 20,000 pairs from 1024^2 bubble-Poisson solves and 512 x 1536 film solves
# (train_solver_pairs); the weights the benchmark's learned legs use
SOLVER_PAIR_WEIGHTS = os.path.join(HERE, "weights", "unet_guess_solver_pairs.npy")


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


def batch_device(rng, gen, count, n, *, bubbles_per_1024sq=64, rmin=8.0, rmax=48.0, rho_in=1000.0):
    """count problems of problem()'s distribution built on the GPU (the numpy builder takes
    about 0.2 s per 1024^2 problem): CUDA tensors rho, f, bx, by of shape (count, n, n) and
    (count, n + 1, n).  rng draws the bubbles, gen (a CUDA torch.Generator) the RHS."""
    import torch
    dev = "cuda"
    xs = torch.arange(n, device=dev, dtype=torch.float64) + 0.5
    rho = torch.ones((count, n, n), device=dev, dtype=torch.float64)
    for i in range(count):
        nb = max(1, int(rng.poisson(bubbles_per_1024sq * n * n / 1024.0 ** 2)))
        cx, cy, rr = rng.uniform(0.0, n, nb), rng.uniform(0.0, n, nb), rng.uniform(rmin, rmax, nb)
        for k in range(nb):
            dx = (xs - float(cx[k])).abs()
            dx = torch.minimum(dx, n - dx)
            dy = xs - float(cy[k])
            rho[i][(dy[:, None] ** 2 + dx[None, :] ** 2) <= float(rr[k]) ** 2] = rho_in
    f = torch.randn((count, n, n), generator=gen, device=dev, dtype=torch.float64)
    f -= f.mean(dim=(1, 2), keepdim=True)
    bx = 2.0 / (rho + torch.roll(rho, 1, dims=2))
    by = torch.empty((count, n + 1, n), device=dev, dtype=torch.float64)
    by[:, 1:n] = 2.0 / (rho[:, 1:] + rho[:, :-1])
    by[:, 0] = 1.0 / rho[:, 0]
    by[:, n] = 1.0 / rho[:, n - 1]
    return rho, f.contiguous(), bx.contiguous(), by


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


def film_pairs(nx, ny, steps, props=None, warm=2):
    """(rho, f, bx, by, dp) pressure systems of the 2-D film step's own solves: a film of nx x ny
    (interface at ny/24 cells, amplitude nx/128 cells -- the 512 x 1536 film's shape at any size) run for
    warm + steps RK3 steps on the GPU; the three substeps' systems of each of the last steps,
    as CUDA tensors (a list of dicts)."""
    import torch
    from . import film2d as G
    P = G.default_props() if props is None else props
    st = G.to_device(G.initial_state(nx, ny, ny / 24.0, nx / 128.0, props=P))
    dt = G.stable_dt(nx, P)
    film = G.Film2D(nx, ny, P)
    buf = torch.zeros(3 * (4 * nx * ny + (ny + 1) * nx), dtype=torch.float64, device="cuda")
    out = []
    try:
        for k in range(warm + steps):
            film.capture(buf if k >= warm else None)
            film.step(st, dt)
            if k >= warm:
                out += [{key: v.clone() for key, v in sysk.items()} for sysk in film.unpack_capture(buf)]
    finally:
        film.capture(None)
        film.close()
    return out


def train_film(net, steps, nx, ny, lr=1e-3, lr_final=1e-4, seed=0, pool_steps=64, log_every=100, log=print):
    """Adam steps of the A-norm loss on the film's own (rho, f -> dp) pairs: a pool of
    3 pool_steps systems from consecutive film steps, net.n drawn per step.  Returns the
    loss history."""
    import torch
    rng = np.random.default_rng(seed)
    pool = film_pairs(nx, ny, pool_steps)
    h = 1.0 / nx
    hist = []
    t0 = time.time()
    for it in range(steps):
        lr_it = lr * (lr_final / lr) ** (it / max(1, steps - 1))
        pick = rng.choice(len(pool), size=net.n, replace=False)
        rho, f, bx, by, dp = (torch.stack([pool[i][k] for i in pick]).contiguous()
                              for k in ("rho", "f", "bx", "by", "dp"))
        loss = net.train_step(rho, f, bx, by, h, h, lr_it, p_star=dp)
        hist.append(loss)
        if log and (it % log_every == 0 or it == steps - 1):
            log(f"film step {it:5d}  loss {np.mean(hist[-log_every:]):.4e}  ({time.time() - t0:.1f} s)")
    return hist


def train_solver_pairs(pairs=20000, n2=1024, film=(512, 1536), images=4, lr=1e-3, lr_final=1e-4, seed=0, chunk=200,
                       log=print, checkpoint=None):
    """The solver-pair training set: (density, RHS -> pressure) pairs from bubble-Poisson solves (n2 x n2,
    the benchmark's bubble distribution built on the GPU, each problem solved to 1e-10 by the
    multigrid) and
    from film solves (the 2-D film step's own three pressure systems per step at its full
    size, captured as the film runs), half each, interleaved in chunks of `chunk` Adam steps.
    One set of weights (the network is dimensionless); each grid shape keeps its own Adam
    moments, and the weights move between the two at every switch (and to `checkpoint`, a
    .npy path, if given).  Returns (params, loss history per source)."""
    import torch
    from . import film2d as G
    from . import poisson
    from .unet import LearnedGuess
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    nx, ny = film
    net2 = LearnedGuess(images, n2, n2, seed=seed + 1)
    net3 = LearnedGuess(3, ny, nx, seed=seed + 1)
    net3.set_params(net2.get_params())
    h2 = 1.0 / n2
    solver = poisson.MultigridPoisson(n2, n2, h2, h2, nlevels=max(2, int(np.log2(n2)) - 4), ncoarse=1)
    P = G.default_props()
    fst = G.to_device(G.initial_state(nx, ny, ny / 24.0, nx / 128.0, props=P))
    fdt = G.stable_dt(nx, P)
    fgpu = G.Film2D(nx, ny, P)
    buf = torch.zeros(3 * (4 * nx * ny + (ny + 1) * nx), dtype=torch.float64, device="cuda")
    steps2 = pairs // 2 // images
    steps3 = pairs // 2 // 3
    total = steps2 + steps3
    hist = {"bubbles": [], "film": []}
    done2 = done3 = 0
    cur = 2
    t0 = time.time()
    try:
        fgpu.step(fst, fdt)     # the film's first step starts from the hydrostatic pressure
        while done2 < steps2 or done3 < steps3:
            if cur == 2 and done2 >= steps2:
                cur = 3
            if cur == 3 and done3 >= steps3:
                cur = 2
            net = net2 if cur == 2 else net3
            for _ in range(chunk):
                it = done2 + done3
                lr_it = lr * (lr_final / lr) ** (it / max(1, total - 1))
                if cur == 2:
                    if done2 >= steps2:
                        break
                    rho, f, bx, by = batch_device(rng, gen, images, n2)
                    ps = torch.zeros_like(f)
                    for i in range(images):
                        _, _, st = solver.solve(ps[i], f[i], bx[i], by[i], rtol=1e-10, max_iters=200)
                        if st != 0:
                            raise RuntimeError(f"solver status {st} on a bubble-Poisson training problem")
                    hist["bubbles"].append(net.train_step(rho, f, bx, by, h2, h2, lr_it, p_star=ps))
                    done2 += 1
                else:
                    if done3 >= steps3:
                        break
                    fgpu.capture(buf)
                    fgpu.step(fst, fdt)
                    fgpu.capture(None)
                    sys3 = fgpu.unpack_capture(buf)
                    rho, f, bx, by, dp = (torch.stack([q[k] for q in sys3]).contiguous()
                                          for k in ("rho", "f", "bx", "by", "dp"))
                    hist["film"].append(net.train_step(rho, f, bx, by, 1.0 / nx, 1.0 / nx, lr_it, p_star=dp))
                    done3 += 1
            other = net3 if cur == 2 else net2
            params = net.get_params()
            other.set_params(params)
            if checkpoint:
                np.save(checkpoint, params)
            if log:
                l2 = np.mean(hist["bubbles"][-50:]) if hist["bubbles"] else 0.0
                l3 = np.mean(hist["film"][-50:]) if hist["film"] else 0.0
                log(f"pairs {images * done2 + 3 * done3:6d}  bubble loss {l2:.4e}  film loss {l3:.4e}  "
                    f"({time.time() - t0:.1f} s)")
            cur = 3 if cur == 2 else 2
        params = (net2 if cur == 3 else net3).get_params()
    finally:
        fgpu.capture(None)
        fgpu.close()
        solver.close()
        net2.close()
        net3.close()
    return params, hist


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
    ap.add_argument("--film", action="store_true",
                    help="train on the 2-D film step's own pressure systems (writes the film weights)")
    ap.add_argument("--film-nx", type=int, default=256)
    ap.add_argument("--solver-pairs", type=int, default=0, metavar="PAIRS",
                    help="train on PAIRS pairs from 1024^2 bubble-Poisson and 512 x 1536 film solves")
    a = ap.parse_args()
    from .unet import LearnedGuess
    if a.solver_pairs:
        params, _ = train_solver_pairs(a.solver_pairs, images=a.batch, lr=a.lr, lr_final=a.lr_final, seed=a.seed)
        os.makedirs(os.path.dirname(a.out), exist_ok=True)
        np.save(a.out, params)
        return
    if a.film:
        nx, ny = a.film_nx, 3 * a.film_nx
        net = LearnedGuess(a.batch, ny, nx, seed=a.seed + 1)
        train_film(net, a.steps, nx, ny, lr=a.lr, lr_final=a.lr_final, seed=a.seed)
        save(net, a.out if a.out != WEIGHTS else FILM_WEIGHTS)
        return
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
