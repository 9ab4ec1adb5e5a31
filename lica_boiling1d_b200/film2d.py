"""2-D film boiling on the GPU (lica_film2d_*): one RK3 time step of the MAC flow grid and the
refined level set, its pressure solves by the 2-D multigrid.

The step generalises the reference's 1-D column step to 2-D (x periodic; y the wall-normal
direction with a heated no-slip wall at the bottom and an outflow top, p = 0 on the top face):
RK3COEF substeps (1d.f:1310-1322), explicit momentum (RHSZ / LHSW's terms, 1d.f:1603-1809),
the projection with the phase-change volume source (PRESSURE_CORRECTION, CAL_CONTINUITY2),
the smeared interfacial mass flux (TEMP_GRAD / TF_GRAD / VOL_TOT_MFDOT, chphase.f), the energy
update (PASSIVE_SCALAR / TEMPASSIGN), TRANSPORT_RK3 with HJWENO and REINITIALIZATION with
GODUNOV (two_phase.f), and surface tension as a continuum surface force with the level set's
curvature (CAL_CUR).  No interface recession term, explicit viscous terms.

Fields (torch CUDA float64, contiguous, x fastest): u (ny, nx) on the face west of each cell,
v (ny + 1, nx) on the face below each cell row, p (the modified pressure p + rho_l g y), th =
(T - T_sat) / dT_wall and phi (2 ny, 2 nx; liquid where phi > 0).
"""
import ctypes as C

import numpy as np

from . import native

FIELDS = ("u", "v", "p", "th", "phi")


def default_props():
    """The 2-D film-boiling benchmark's liquid/vapour ratios (Welch and Wilson's case: rho 200/5,
    mu 0.1/0.005, k 40/1, c_p 400/200, h_fg 1e4, superheat 5 K): density 40, viscosity 20,
    conductivity 40, specific heat 2, Ja = c_p,v dT / h_fg = 0.1, Pr_v = 1, and Re = 69.2 and
    Fr = 1 on the velocity sqrt(g Lx) with Lx the most dangerous Rayleigh-Taylor wavelength
    (0.0787 m), We = rho_v U^2 Lx / sigma = 3.04 (sigma 0.1 N/m).  The pressure solves stop at
    a relative residual of 1e-10, or at FP64's attainable accuracy where that lies above it
    (LICA_STALLED): at 512 x 1536 the phase-change source leaves a pressure increment so large
    against its right-hand side (||A|| ||dp|| / ||f|| ~ 1e7) that rounding the exact increment to
    FP64 alone gives a relative residual of 1.6e-10, and the solves end near 3e-10 after about
    12 iterations.  At 64 x 192 the floor is 6e-12 and 1e-10 is met in 9."""
    return dict(re=69.2, visr=20.0, denr=40.0, prm=1.0, scr=2.0, tcr=40.0, jakob=0.1, fr=1.0, we=3.04,
                rtol=1e-10, nreinit=2)


def initial_state(nx, ny, y0_cells=64.0, amp_cells=4.0, props=None):
    """The film: interface y = y0 h + amp h cos(2 pi x) (Lx = 1, h = 1/nx), phi = y - y_i(x) on
    the refined centres (liquid where phi > 0); theta linear in the vapour from 1 at the wall to
    0 at the interface and 0 in the liquid; u = v = 0; p the discrete hydrostatic (modified)
    pressure of the initial density field, which balances the buoyancy g (rho_l / rho_f - 1) on
    every face with the projection's own face density rho_f = (rho_below + rho_above) / 2 (top
    face: p = 0 half a cell above the last row), so the first pressure solve starts from the
    balanced state.  Host numpy arrays."""
    h = 1.0 / nx
    hf = 0.5 * h
    xf = (np.arange(2 * nx) + 0.5) * hf
    yf = (np.arange(2 * ny) + 0.5) * hf
    yi_f = y0_cells * h + amp_cells * h * np.cos(2.0 * np.pi * xf)
    phi = np.ascontiguousarray(yf[:, None] - yi_f[None, :])
    xc = (np.arange(nx) + 0.5) * h
    yc = (np.arange(ny) + 0.5) * h
    yi_c = y0_cells * h + amp_cells * h * np.cos(2.0 * np.pi * xc)
    th = np.maximum(0.0, 1.0 - yc[:, None] / yi_c[None, :])
    z = np.zeros((ny, nx))
    P = default_props() if props is None else props
    g = 0.0 if P["fr"] == 0.0 else 1.0 / (P["fr"] * P["fr"])
    denp = P["denr"]
    # density per cell from the smoothed Heaviside of phi (the step's property rule)
    eps = h
    s = (phi + eps) * (1.0 / (2.0 * eps))
    H = np.where(phi <= -eps, 0.0, np.where(phi >= eps, 1.0, s * s * s * (10.0 + s * (-15.0 + 6.0 * s))))
    psi = 0.25 * ((H[0::2, 0::2] + H[0::2, 1::2]) + (H[1::2, 0::2] + H[1::2, 1::2]))
    den = 1.0 + (denp - 1.0) * psi
    p = np.zeros((ny, nx))
    p[ny - 1] = 0.0 - (0.5 * h) * (g * (denp - den[ny - 1]))
    for j in range(ny - 1, 0, -1):
        p[j - 1] = p[j] - h * (g * (denp - 0.5 * (den[j - 1] + den[j])))
    return dict(u=z.copy(), v=np.zeros((ny + 1, nx)), p=p, th=th, phi=phi)


def stable_dt(nx, props, cfl=0.2):
    """cfl times the smallest explicit limit from rest: viscous and thermal diffusion of the
    faster-diffusing phase and the gravity wave time sqrt(h / g)."""
    P = props
    h = 1.0 / nx
    nu = max(1.0 / P["re"], (P["visr"] / P["re"]) / P["denr"])
    al = (1.0 / (P["re"] * P["prm"])) * max(1.0, P["tcr"] / (P["denr"] * P["scr"]))
    lim = [0.25 * h * h / nu, 0.25 * h * h / al]
    g = 0.0 if P["fr"] == 0.0 else 1.0 / (P["fr"] * P["fr"])
    if g > 0.0:
        lim.append(float(np.sqrt(h / g)))
    return cfl * min(lim)


def levels_for(nx, ny, coarsest=16):
    """Multigrid levels down to a coarsest level of at least `coarsest` cells per side."""
    lv = 1
    while nx % 2 == 0 and ny % 2 == 0 and min(nx, ny) // 2 >= coarsest and (nx // 2) % 16 == 0 and \
            (ny // 2) % 16 == 0:
        nx //= 2
        ny //= 2
        lv += 1
    return lv


def to_device(state):
    import torch
    return {k: torch.from_numpy(np.ascontiguousarray(state[k], dtype=np.float64)).cuda() for k in FIELDS}


def to_host(state):
    return {k: state[k].cpu().numpy() for k in FIELDS}


class Film2D:
    """The GPU step for an nx x ny grid (multiples of 32): step(state, dt) advances the device
    fields in place and returns the pressure solves' iterations and residuals."""

    def __init__(self, nx, ny, props=None, *, nlevels=None, precision="fp64", max_iters=200):
        self.nx, self.ny = nx, ny
        self.props = dict(default_props() if props is None else props)
        P = self.props
        self._p = native.Film2DProps(re=P["re"], visr=P["visr"], denr=P["denr"], prm=P["prm"], scr=P["scr"],
                                     tcr=P["tcr"], jakob=P["jakob"], fr=P["fr"], we=P.get("we", 0.0), rtol=P["rtol"],
                                     max_iters=max_iters, nreinit=int(P["nreinit"]))
        self.nlevels = levels_for(nx, ny) if nlevels is None else nlevels
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision is 'fp64' or 'mixed'")
        h = C.c_void_p()
        native.check(native.lib().lica_film2d_create(C.byref(h), nx, ny, C.byref(self._p), self.nlevels,
                                                     0 if precision == "fp64" else 1), "lica_film2d_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            native.lib().lica_film2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, state, dt, stream=None):
        import torch
        shapes = dict(u=(self.ny, self.nx), v=(self.ny + 1, self.nx), p=(self.ny, self.nx), th=(self.ny, self.nx),
                      phi=(2 * self.ny, 2 * self.nx))
        for k in FIELDS:
            t = state[k]
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and tuple(t.shape) == shapes[k]):
                raise ValueError(f"{k}: contiguous CUDA float64 of shape {shapes[k]} expected")
        s = stream if stream is not None else torch.cuda.current_stream()
        st = native.Film2DStats()
        code = native.lib().lica_film2d_step_device(self._h, *(state[k].data_ptr() for k in FIELDS), float(dt),
                                                    C.byref(st), s.cuda_stream)
        native.check(code, "lica_film2d_step_device", ok=(0, 1, 8))
        return dict(iterations=list(st.iterations), status=list(st.status), rel=list(st.rel_residual),
                    guess_rel=list(st.guess_rel), code=code)

    def set_guess(self, net):
        """Start the three pressure solves from the learned guess of net (a LearnedGuess of
        one ny x nx image; zero where the guess is no better than zero); None: from zero."""
        if net is not None and (net.n, net.h, net.w) != (1, self.ny, self.nx):
            raise ValueError(f"the guess must be a LearnedGuess(1, {self.ny}, {self.nx})")
        self._guess = net   # keep it alive while attached
        native.check(native.lib().lica_film2d_set_guess(self._h, net._h if net is not None else None),
                     "lica_film2d_set_guess")

    def warm_start(self, on=True):
        """Start each substep's pressure solve from the increment the same substep solved in
        the previous step (zero in the first step); the kept increments are forgotten."""
        native.check(native.lib().lica_film2d_set_warm_start(self._h, 1 if on else 0), "lica_film2d_set_warm_start")

    def capture(self, systems):
        """Record every step's three pressure systems into systems, a float64 CUDA tensor of
        3 * (4 nx ny + (ny + 1) nx) values (per substep: density, f, bx, by, dp); None: off."""
        if systems is not None and systems.numel() < 3 * (4 * self.nx * self.ny + (self.ny + 1) * self.nx):
            raise ValueError("capture buffer too small")
        self._systems = systems
        native.check(native.lib().lica_film2d_capture_device(
            self._h, C.c_void_p(systems.data_ptr()) if systems is not None else None), "lica_film2d_capture_device")

    def unpack_capture(self, systems):
        """The captured systems as a list of 3 dicts of (ny, nx) / (ny + 1, nx) tensors."""
        n, nb = self.nx * self.ny, (self.ny + 1) * self.nx
        out = []
        for k in range(3):
            q = systems[k * (4 * n + nb):(k + 1) * (4 * n + nb)]
            out.append(dict(rho=q[:n].view(self.ny, self.nx), f=q[n:2 * n].view(self.ny, self.nx),
                            bx=q[2 * n:3 * n].view(self.ny, self.nx), by=q[3 * n:3 * n + nb].view(self.ny + 1, self.nx),
                            dp=q[3 * n + nb:4 * n + nb].view(self.ny, self.nx)))
        return out

    def mdot(self, stream=None):
        """The interfacial mass flux per cell of the last substep, (ny, nx) on the device."""
        import torch
        out = torch.empty((self.ny, self.nx), dtype=torch.float64, device="cuda")
        s = stream if stream is not None else torch.cuda.current_stream()
        native.check(native.lib().lica_film2d_mdot_device(self._h, out.data_ptr(), s.cuda_stream),
                     "lica_film2d_mdot_device")
        return out
