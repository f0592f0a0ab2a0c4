"""Reaction-network definitions used by the tests, the bench and the examples.

A model is a box 0 <= x_s <= b_s, a stoichiometry nu[r, s] (net change of species s when reaction
r fires) and a factorised propensity a_r(x) = c_r(t) * prod_s f_{r,s}(x_s).  The per-species
factor tables f_{r,s}(0..b_s) have the layout of the reference's SDKronMatSet::vals
(src/fspmat_kron_kernels.cu:170-190: reaction-major, then species, then x_s); the coefficients
c_r(t) play the part of the reference's TcoefFun (src/FSPMat.h:16).

Workloads (synthetic, seeded):
  toggle(bounds)   two-gene toggle switch of the reference tests (tests/test_fsp_mat.cu:19-97)
  birth_death_2    2 species, 4 mass-action reactions, box 127 x 255 (32,768 states)
  gene_expression  5 species (3 binary genes, nuclear and cytoplasmic mRNA), 12 reactions,
                   box 1x1x1x127x127 (131,072 states), one switching rate k0*sigmoid((t-5)/0.5)
  mass_action_3    3 species, 9 mass-action reactions, rates log-uniform in [1e-2, 10] from seed
                   20261203, box 255^3 (16,777,216 states), p0 = Poisson(5)^3
  gene_batch       parameter sets of gene_expression with uneven boxes (batched solves)
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable

import numpy as np


@dataclass
class CMEModel:
    name: str
    bounds: list[int]
    nu: np.ndarray                       # [nr, ns] int32 net stoichiometry
    tables: np.ndarray                   # [nr, sum(b_s + 1)] float64 factor tables
    rates: np.ndarray                    # [nr] float64 time-invariant coefficients c_r
    tcoef: Callable[[float], np.ndarray] | None = None   # c(t); None -> rates
    p0_kind: str = "delta0"              # "delta0" | "poisson5"
    meta: dict = field(default_factory=dict)
    factor: Callable[[int, int, int], float] | None = None  # f_{r,s}(x) for any x (boxes of any size)

    @property
    def ns(self) -> int:
        return len(self.bounds)

    @property
    def nr(self) -> int:
        return int(self.nu.shape[0])

    @property
    def n_states(self) -> int:
        return int(np.prod([b + 1 for b in self.bounds], dtype=np.int64))

    def coefs(self, t: float = 0.0) -> np.ndarray:
        if self.tcoef is None:
            return self.rates.copy()
        return np.asarray(self.tcoef(t), dtype=np.float64)

    def stoich_csr(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Stoichiometry as the reference's CSRMatInt (rows = reactions, cols = species)."""
        vals, cols, rows = [], [], [0]
        for r in range(self.nr):
            for s in range(self.ns):
                if self.nu[r, s] != 0:
                    vals.append(int(self.nu[r, s]))
                    cols.append(s)
            rows.append(len(vals))
        return (np.asarray(vals, np.int32), np.asarray(cols, np.int32), np.asarray(rows, np.int32))

    def p0(self) -> np.ndarray:
        n = self.n_states
        if self.p0_kind == "delta0":
            p = np.zeros(n)
            p[0] = 1.0
            return p
        if self.p0_kind == "poisson5":
            p = np.ones(1)
            for b in self.bounds:  # species 0 fastest: kron(p_last, ..., p_0)
                k = np.arange(b + 1)
                lp = k * math.log(5.0) - 5.0 - np.array([math.lgamma(v + 1.0) for v in k])
                p = np.kron(np.exp(lp), p)
            return p
        raise ValueError(self.p0_kind)


def _tables_from(bounds, nr, fn) -> np.ndarray:
    """fn(x, species, reaction) -> f_{r,s}(x); filled in the reference order."""
    stride = sum(b + 1 for b in bounds)
    t = np.empty((nr, stride))
    for r in range(nr):
        off = 0
        for s, b in enumerate(bounds):
            x = np.arange(b + 1, dtype=np.float64)
            t[r, off:off + b + 1] = fn(x, s, r)
            off += b + 1
    return t


def mass_action(bounds, nu, orders, rates, name="mass_action", tcoef=None, p0_kind="delta0", meta=None) -> CMEModel:
    """Propensity c_r * prod_s C(x_s, m_{r,s}) * m_{r,s}! = c_r * prod_s x_s (x_s-1) .. (x_s-m+1)."""
    nu = np.asarray(nu, np.int32)
    orders = np.asarray(orders, np.int32)

    def fn(x, s, r):
        m = int(orders[r, s])
        v = np.ones_like(x)
        for j in range(m):
            v = v * np.maximum(x - j, 0.0)
        return v

    tables = _tables_from(bounds, nu.shape[0], fn)

    def factor(x, s, r):  # the same falling factorial for a single count
        v = 1.0
        for j in range(int(orders[r, s])):
            v *= max(x - j, 0.0)
        return v
    return CMEModel(name, list(bounds), nu, tables, np.asarray(rates, np.float64), tcoef, p0_kind, meta or {}, factor)


# ---- the reference's toggle switch (tests/test_fsp_mat.cu:19-97, test_kry_expv.cu:80-106) ----
TOGGLE = dict(ayx=2.6e-3, axy=6.1e-3, nyx=3e0, nxy=2.1e0, kx0=2.2e-3, kx=1.7e-2, dx=3.8e-4,
              ky0=6.8e-5, ky=1.6e-2, dy=3.8e-4)


def toggle(bounds=(31, 31), time_varying=False) -> CMEModel:
    p = TOGGLE
    nu = np.array([[1, 0], [1, 0], [-1, 0], [0, 1], [0, 1], [0, -1]], np.int32)

    def hill(x, a, h):  # math.pow is the C library pow, as in the reference's factor function
        return np.array([1.0 / (1.0 + a * math.pow(float(v), h)) for v in x])

    def fn(x, s, r):  # toggle_propensity_factor, tests/test_fsp_mat.cu:52-84
        one = np.ones_like(x)
        if r == 1 and s == 1:
            return hill(x, p["ayx"], p["nyx"])
        if r == 2 and s == 0:
            return x.copy()
        if r == 4 and s == 0:
            return hill(x, p["axy"], p["nxy"])
        if r == 5 and s == 1:
            return x.copy()
        return one

    rates = np.array([p["kx0"], p["kx"], p["dx"], p["ky0"], p["ky"], p["dy"]])
    tcoef = None
    if time_varying:  # tests/test_sundials.cu:55-64
        def tcoef(t):
            return np.array([p["kx0"], p["kx"] * (1.0 + math.cos(t / 1000.0)), p["dx"] * math.exp(-t / 3600.0),
                             p["ky0"], p["ky"], p["dy"] * math.exp(-t / 3600.0)])
    def factor(x, s, r):
        return float(fn(np.array([float(x)]), s, r)[0])
    return CMEModel("toggle", list(bounds), nu, _tables_from(bounds, 6, fn), rates, tcoef, factor=factor)


def birth_death_2() -> CMEModel:
    """2 species, 4 reactions: 0->S1 (10), S1->0 (1.0 x1), 0->S2 (0.5 x1), S2->0 (0.2 x2)."""
    nu = [[1, 0], [-1, 0], [0, 1], [0, -1]]
    orders = [[0, 0], [1, 0], [1, 0], [0, 1]]
    return mass_action((127, 255), nu, orders, [10.0, 1.0, 0.5, 0.2], name="birth_death_2")


GENE = dict(k_on=(0.05, 0.04, 0.03), k_off=(2.0, 2.0, 3.0), k_tx=(5.0, 15.0, 50.0), k_exp=0.5, g_n=0.1, g_c=0.05,
            k0=0.1)


def gene_expression(bounds=(1, 1, 1, 127, 127), time_varying=True, rates_scale=None) -> CMEModel:
    """3 binary genes g1..g3, nuclear n and cytoplasmic c mRNA.  Reactions:
    0-2  gene i on  (rate k_on_i * (1 - g_i)); reaction 0 uses k0 * sigmoid((t - 5) / 0.5) when time_varying
    3-5  gene i off (rate k_off_i * g_i)
    6-8  transcription from gene i: 0 -> n at k_tx_i * g_i
    9    export n -> c at 0.5 n;  10  n -> 0 at 0.1 n;  11  c -> 0 at 0.05 c."""
    g = GENE
    ns = 5
    nu = np.zeros((12, ns), np.int32)
    for i in range(3):
        nu[i, i] = 1
        nu[3 + i, i] = -1
        nu[6 + i, 3] = 1
    nu[9, 3], nu[9, 4] = -1, 1
    nu[10, 3] = -1
    nu[11, 4] = -1

    def fn(x, s, r):
        one = np.ones_like(x)
        if r < 3 and s == r:
            return 1.0 - x
        if 3 <= r < 6 and s == r - 3:
            return x.copy()
        if 6 <= r < 9 and s == r - 6:
            return x.copy()
        if r in (9, 10) and s == 3:
            return x.copy()
        if r == 11 and s == 4:
            return x.copy()
        return one

    rates = np.array(list(g["k_on"]) + list(g["k_off"]) + list(g["k_tx"]) + [g["k_exp"], g["g_n"], g["g_c"]])
    if rates_scale is not None:
        rates = rates * np.asarray(rates_scale)
    tcoef = None
    if time_varying:
        base = rates.copy()

        def tcoef(t):
            c = base.copy()
            c[0] = g["k0"] / (1.0 + math.exp(-(t - 5.0) / 0.5))
            return c
    return CMEModel("gene_expression", list(bounds), nu, _tables_from(bounds, 12, fn), rates, tcoef)


def mass_action_3(bound=255, seed=20261203, bounds=None) -> CMEModel:
    """3 species, 9 mass-action reactions with log-uniform rates in [1e-2, 10] (seeded):
    0->S1, 0->S2, S1->0, S2->0, S3->0, S1->S2, S2->S3, S1+S2->S1+S2+S3 (x1 x2), S1+S3->S1 (x1 x3).
    The box is bound^3, or `bounds` when given."""
    rng = np.random.default_rng(seed)
    rates = 10.0 ** rng.uniform(-2.0, 1.0, size=9)
    nu = [[1, 0, 0], [0, 1, 0], [-1, 0, 0], [0, -1, 0], [0, 0, -1], [-1, 1, 0], [0, -1, 1], [0, 0, 1], [0, 0, -1]]
    orders = [[0, 0, 0], [0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 0, 0], [0, 1, 0], [1, 1, 0], [1, 0, 1]]
    b = tuple(bounds) if bounds is not None else (bound, bound, bound)
    return mass_action(b, nu, orders, rates, name="mass_action_3", p0_kind="poisson5", meta={"seed": seed})


def gene_batch(n: int = 256, seed: int = 20261204, lo: int = 63, hi: int = 255) -> list[CMEModel]:
    """n parameter sets of gene_expression with time-invariant rates: every rate log-uniform within
    one decade of its nominal value, nuclear and cytoplasmic mRNA bounds uniform in lo..hi."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        scale = 10.0 ** rng.uniform(-1.0, 1.0, size=12)
        bn, bc = (int(v) for v in rng.integers(lo, hi + 1, size=2))
        out.append(gene_expression((1, 1, 1, bn, bc), time_varying=False, rates_scale=scale))
    return out
