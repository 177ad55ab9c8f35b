"""Generates the golden fixtures of tests/golden/ (test infrastructure).

The reference (jojo240607/physics, Rust) cannot be compiled in this
environment and its own tests contain no golden vectors for the SPH step, so
the fixtures come from this file: a second, pure-Python restatement of
FluidWorld<f64>::step, written separately from the C++ oracle and following
the reference source line by line:

  crates/phy-fluid/src/kernels.rs:22-65      kernel coefficients and kernels
  crates/phy-fluid/src/sph/grid.rs:25-56     cell keys and neighbour order
  crates/phy-fluid/src/sph/world.rs:124-169  fill_box, lattice_mass
  crates/phy-fluid/src/sph/world.rs:183-397  step: density, forces,
                                             integrate, bounds

Python floats are IEEE doubles and Python never fuses a*b+c, so evaluating
the reference's expressions in the reference's order reproduces its f64
results bit for bit (math.pow is the C library pow, as Rust's powf).

Run:  python tests/golden/gen_golden.py   (writes *.npz next to this file)
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def defaults():
    # SphParams::defaults() (params.rs:55-85)
    return dict(rest_density=1000.0, stiffness=250.0, viscosity=3.5, visc_k=[3.5], visc_n=[1.0], shear_min=0.01,
                mass=0.02, h=0.2, gravity=(0.0, -9.81, 0.0), bounds_min=(-5.0, -5.0, -5.0),
                bounds_max=(5.0, 5.0, 5.0), boundary_damp=0.4, xsph_eps=0.5)


class Kernels:
    def __init__(self, h):
        pi = math.pi
        self.h = h
        self.h2 = h * h
        h3 = self.h2 * h
        h6 = h3 * h3
        h9 = h6 * h3
        self.poly6_coeff = 315.0 / (64.0 * pi * h9)
        self.spiky_grad_coeff = -45.0 / (pi * h6)
        self.visc_lap_coeff = 45.0 / (pi * h6)

    def poly6(self, r):
        if r >= self.h:
            return 0.0
        diff = self.h2 - r * r
        return self.poly6_coeff * diff * diff * diff

    def spiky_grad_mag(self, r):
        if r >= self.h or r <= 0.0:
            return 0.0
        diff = self.h - r
        return self.spiky_grad_coeff * diff * diff

    def visc_lap(self, r):
        if r >= self.h:
            return 0.0
        return self.visc_lap_coeff * (self.h - r)


def norm(v):
    return math.sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])


def to_i64(x):
    if x != x or not (-9223372036854775808.0 < x < 9223372036854775808.0):
        return 0
    return int(x)


class World:
    def __init__(self, params):
        self.params = dict(params)
        self.h0 = params["h"]
        self.k = Kernels(self.h0)
        self.cell = self.h0
        self.ps = []  # dicts: pos, vel, acc, body_acc, rho, p, mass, material, mu_eff, xsph

    def key_of(self, p):
        inv = 1.0 / self.cell
        return tuple(to_i64(math.floor(p[a] * inv)) for a in range(3))

    def lattice_mass(self, s):
        h = self.params["h"]
        n_shell = int(math.ceil(h / s)) + 1
        sum_w = 0.0
        for i in range(-n_shell, n_shell + 1):
            for j in range(-n_shell, n_shell + 1):
                for l in range(-n_shell, n_shell + 1):
                    rr = math.sqrt(float(i * i + j * j + l * l))
                    r = s * rr
                    if r < h:
                        sum_w += self.k.poly6(r)
        return self.params["rest_density"] / sum_w if sum_w > 0.0 else self.params["mass"]

    def add(self, pos, mass, vel=(0.0, 0.0, 0.0), material=0):
        self.ps.append(dict(pos=list(pos), vel=list(vel), acc=[0.0, 0.0, 0.0], body_acc=[0.0, 0.0, 0.0], rho=0.0,
                            p=0.0, mass=mass, material=material, mu_eff=0.0, xsph=[0.0, 0.0, 0.0]))

    def fill_box(self, mn, mx, spacing, margin):
        lo = [mn[a] + margin for a in range(3)]
        hi = [mx[a] - margin for a in range(3)]
        d = spacing
        mass = self.lattice_mass(d)
        x = lo[0]
        while x <= hi[0]:
            y = lo[1]
            while y <= hi[1]:
                z = lo[2]
                while z <= hi[2]:
                    self.add((x, y, z), mass)
                    z += d
                y += d
            x += d

    def neighbors(self, grid, p):
        ci, cj, ck = self.key_of(p)
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                for dk in (-1, 0, 1):
                    for j in grid.get((ci + di, cj + dj, ck + dk), ()):
                        yield j

    def step(self, dt):
        ps = self.ps
        if not ps:
            return
        grid = {}
        for i, pt in enumerate(ps):
            grid.setdefault(self.key_of(pt["pos"]), []).append(i)
        prm = self.params
        h = prm["h"]
        k = self.k
        pos = [list(pt["pos"]) for pt in ps]
        mass = [pt["mass"] for pt in ps]
        rho_out, p_out = [], []
        for i in range(len(ps)):
            p_i = pos[i]
            rho = 0.0
            for j in self.neighbors(grid, p_i):
                r = norm([p_i[a] - pos[j][a] for a in range(3)])
                if r < h:
                    rho += mass[j] * k.poly6(r)
            over = rho - prm["rest_density"]
            p = prm["stiffness"] * over if over > 0.0 else 0.0
            rho_out.append(rho)
            p_out.append(p)
        for i, pt in enumerate(ps):
            pt["rho"] = rho_out[i]
            pt["p"] = p_out[i]
        vel = [list(pt["vel"]) for pt in ps]
        rho = [pt["rho"] for pt in ps]
        pr = [pt["p"] for pt in ps]
        res = []
        for i in range(len(ps)):
            p_i, v_i, rho_i, p_i_p, m_i = pos[i], vel[i], rho[i], pr[i], mass[i]
            f_press = [0.0, 0.0, 0.0]
            f_visc_raw = [0.0, 0.0, 0.0]
            xsph = [0.0, 0.0, 0.0]
            shear = 0.0
            for j in self.neighbors(grid, p_i):
                if j == i:
                    continue
                d = [pos[j][a] - p_i[a] for a in range(3)]
                r = norm(d)
                if r >= h or r <= 0.0:
                    continue
                rho_j = rho[j]
                p_j = pr[j]
                grad = k.spiky_grad_mag(r)
                dir_ = [d[a] / r for a in range(3)]
                coef = m_i * mass[j] * (p_i_p / (rho_i * rho_i) + p_j / (rho_j * rho_j))
                for a in range(3):
                    f_press[a] += dir_[a] * (coef * grad)
                lap = k.visc_lap(r)
                dv = [vel[j][a] - v_i[a] for a in range(3)]
                s = m_i * mass[j] / rho_j * lap
                for a in range(3):
                    f_visc_raw[a] += dv[a] * s
                w = k.poly6(r)
                s2 = mass[j] / rho_j * w
                for a in range(3):
                    xsph[a] += dv[a] * s2
                shear += norm(dv) / (r + 1e-4) * (mass[j] / rho_j)
            mi = ps[i]["material"]
            m_idx = mi if mi < len(prm["visc_k"]) else 0
            kc = prm["visc_k"][m_idx]
            nn = prm["visc_n"][m_idx]
            sreg = shear if shear > prm["shear_min"] else prm["shear_min"]
            mu_eff = kc * math.pow(sreg, nn - 1.0)
            f_visc = [f_visc_raw[a] * mu_eff for a in range(3)]
            if rho_i > 0.0:
                acc = [(f_press[a] + f_visc[a]) / rho_i for a in range(3)]
            else:
                acc = [0.0, 0.0, 0.0]
            res.append((acc, mu_eff, xsph))
        for i, pt in enumerate(ps):
            pt["acc"], pt["mu_eff"], pt["xsph"] = res[i]
        g = prm["gravity"]
        eps = prm["xsph_eps"]
        for pt in ps:
            a = [(pt["acc"][q] + g[q]) + pt["body_acc"][q] for q in range(3)]
            for q in range(3):
                pt["vel"][q] += a[q] * dt
            for q in range(3):
                pt["vel"][q] += pt["xsph"][q] * eps
            for q in range(3):
                pt["pos"][q] += pt["vel"][q] * dt
            pt["body_acc"] = [0.0, 0.0, 0.0]
        lo, hi, damp = prm["bounds_min"], prm["bounds_max"], prm["boundary_damp"]
        for pt in ps:
            for q in range(3):
                if pt["pos"][q] < lo[q]:
                    pt["pos"][q] = lo[q]
                    pt["vel"][q] = -pt["vel"][q] * damp
                elif pt["pos"][q] > hi[q]:
                    pt["pos"][q] = hi[q]
                    pt["vel"][q] = -pt["vel"][q] * damp

    def snapshot(self):
        f = lambda k: np.array([pt[k] for pt in self.ps], np.float64)
        return dict(pos=f("pos"), vel=f("vel"), acc=f("acc"), rho=f("rho"), p=f("p"), mu_eff=f("mu_eff"),
                    xsph=f("xsph"), mass=f("mass"))


def splitmix_u01(seed, count):
    out = []
    state = seed
    mask = (1 << 64) - 1
    for _ in range(count):
        state = (state + 0x9E3779B97F4A7C15) & mask
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z = z ^ (z >> 31)
        out.append((z >> 11) / float(1 << 53))
    return out


def case_quickstart():
    """README quick start: fill_box((-1,1,-1),(1,3,1),0.3,0.1), dt 0.01, 200 steps."""
    w = World(defaults())
    w.fill_box((-1.0, 1.0, -1.0), (1.0, 3.0, 1.0), 0.3, 0.1)
    first = None
    snaps = {}
    for s in range(200):
        w.step(0.01)
        if s == 0:
            first = w.snapshot()
        if s + 1 in (50, 100, 200):
            snaps[s + 1] = w.snapshot()
    out = {f"step1_{k}": v for k, v in first.items()}
    for n, sn in snaps.items():
        out[f"step{n}_pos"] = sn["pos"]
        out[f"step{n}_vel"] = sn["vel"]
    out["step200_rho"] = snaps[200]["rho"]
    out["step200_acc"] = snaps[200]["acc"]
    np.savez_compressed(HERE / "quickstart.npz", **out)


def jittered_block(nx, ny, nz, s=0.1, seed=0xC0FFEE):
    u = splitmix_u01(seed, 3 * nx * ny * nz)
    pos = []
    q = 0
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                base = ((i + 0.5) * s, (j + 0.5) * s, (k + 0.5) * s)
                pos.append(tuple(base[a] + (2.0 * u[q + a] - 1.0) * (0.05 * s) for a in range(3)))
                q += 3
    return pos


def case_dam216():
    """6x6x6 jittered lattice (spacing h/2), bounds [0,1.2]^3, dt 0.005, 30 steps."""
    prm = defaults()
    prm["bounds_min"] = (0.0, 0.0, 0.0)
    prm["bounds_max"] = (1.2, 1.2, 1.2)
    w = World(prm)
    m = w.lattice_mass(0.1)
    pos = jittered_block(6, 6, 6)
    for p in pos:
        w.add(p, m)
    out = {"init_pos": np.array(pos, np.float64), "mass": np.float64(m)}
    for s in range(30):
        w.step(0.005)
        if s == 0:
            out.update({f"step1_{k}": v for k, v in w.snapshot().items()})
    sn = w.snapshot()
    for k in ("pos", "vel", "rho", "p", "acc", "mu_eff", "xsph"):
        out[f"step30_{k}"] = sn[k]
    np.savez_compressed(HERE / "dam216.npz", **out)


def case_materials():
    """Reference test material_tag_distinguishes_viscosity (sph/tests.rs:406-427) and
    the shear-thinning / thickening configuration (tests.rs:370-404)."""
    prm = defaults()
    prm["bounds_min"] = (-3.0, -3.0, -3.0)
    prm["bounds_max"] = (3.0, 3.0, 3.0)
    prm["gravity"] = (0.0, 0.0, 0.0)
    out = {}
    w = World(prm)
    w.add((0.0, 0.0, 0.0), 0.05, (-300.0, 0.0, 0.0), 0)
    w.add((0.0, 0.06, 0.0), 0.05, (300.0, 0.0, 0.0), 1)
    w.params["visc_k"] = [3.5, 10.0]
    w.params["visc_n"] = [1.0, 1.0]
    w.step(0.001)
    sn = w.snapshot()
    for k in ("pos", "vel", "mu_eff", "acc", "rho"):
        out[f"twomat_{k}"] = sn[k]
    for n in (0.5, 1.0, 1.5):
        w = World(prm)
        for iy in range(2):
            vy = -300.0 if iy == 0 else 300.0
            for ix in range(5):
                w.add(((ix - 2.0) * 0.08, iy * 0.06, 0.0), 0.05, (vy, 0.0, 0.0), 0)
        w.params["visc_k"] = [3.5]
        w.params["visc_n"] = [n]
        w.step(0.001)
        sn = w.snapshot()
        tag = str(n).replace(".", "p")
        out[f"shear{tag}_mu_eff"] = sn["mu_eff"]
        out[f"shear{tag}_pos"] = sn["pos"]
        out[f"shear{tag}_vel"] = sn["vel"]
    np.savez_compressed(HERE / "materials.npz", **out)


if __name__ == "__main__":
    case_quickstart()
    case_dam216()
    case_materials()
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))
