"""Moment-tensor basis of a level, built from the level alone (no template).

The reference builds its basis by enumerating contractions of basic moment
tensors M_{mu,nu} = sum_j f_mu(r_j) u_j^(x nu) (moment_jax.py:116-212): every
multiset of at most four moments (mu, nu) whose level sum(2 + 4 mu + nu) is
within the limit, every binary tree of pairwise tensor contractions over them
that ends in a scalar, and, per multiset, one tree for each distinct scalar
function (functions told apart by their values on test vectors; among trees of
equal value the one with the smallest summed intermediate rank).  It evaluates
that basis with dense 3^nu tensors and maps MLIP coefficients onto it by value
(conversion.py:105-198).

This engine evaluates MLIP tables (alpha_index_basic, alpha_index_times,
alpha_moment_mapping), so here the same enumeration ends in such tables:

* a tensor is a list of axis groups, symmetric within each group (a basic
  moment is one group of nu axes; a contraction keeps the free remainder of
  each operand's groups, left operand first), and a component is one monomial
  (x^a y^b z^c) per group;
* a contraction takes the first n axes of its left operand (as the reference
  does) and any n axes of the right one; only how many axes of each left group
  meet each right group matters (a count matrix), so candidates are count
  matrices, not axis permutations;
* each component of a contraction is a sum over the monomials of the contracted
  axes, sum_c multinomial(c) L[.. + c] R[c + ..], which gives MLIP entries
  m[C] += mult * m[L] * m[R] with integer multiplicities.

`build_basis(level)` returns the tables; `template_potential(...)` wraps them in
an untrained `.mtp` potential the engine loads like a template file.
"""

from __future__ import annotations

import itertools
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

Group = Tuple[int, ...]           # sizes of the symmetric axis groups of a tensor
Node = tuple                      # ("b", mu, nu) or ("c", left, right, counts)

DEFAULT_MAX_MOMENTS = 4


def level_of(mu: int, nu: int) -> int:
    """Level of the basic moment M_{mu,nu}: 2 + 4 mu + nu."""
    return 2 + 4 * mu + nu


def groups_of(node: Node) -> Group:
    """Axis groups of a node (in axis order)."""
    if node[0] == "b":
        return (node[2],) if node[2] > 0 else ()
    _, left, right, counts = node
    lg, rg = groups_of(left), groups_of(right)
    out = [g - sum(row) for g, row in zip(lg, counts)]
    out += [h - sum(counts[i][j] for i in range(len(lg))) for j, h in enumerate(rg)]
    return tuple(s for s in out if s > 0)


def rank_of(node: Node) -> int:
    return sum(groups_of(node))


def _prefix_rows(lg: Group, n: int) -> Optional[Tuple[int, ...]]:
    """How many of the first n axes of a tensor with groups lg fall in each group."""
    rows, left = [], n
    for g in lg:
        take = min(g, left)
        rows.append(take)
        left -= take
    return tuple(rows) if left == 0 else None


def _matrices(rows: Sequence[int], cols: Group):
    """Count matrices with the given row sums and column sums at most cols."""
    if not rows:
        yield ()
        return
    first, rest = rows[0], rows[1:]

    def splits(total, caps):
        if not caps:
            if total == 0:
                yield ()
            return
        for k in range(min(total, caps[0]) + 1):
            for tail in splits(total - k, caps[1:]):
                yield (k,) + tail

    for row in splits(first, list(cols)):
        remaining = tuple(c - k for c, k in zip(cols, row))
        for tail in _matrices(rest, remaining):
            yield (row,) + tail


def contractions(left: Node, right: Node) -> List[Node]:
    """Every contraction of left with right over n >= 1 axes (n >= 0 when either
    is a scalar): the first n axes of left against any n axes of right, one
    node per count matrix."""
    lg, rg = groups_of(left), groups_of(right)
    lr, rr = sum(lg), sum(rg)
    n_min = 0 if lr == 0 or rr == 0 else 1
    out = []
    for n in range(n_min, min(lr, rr) + 1):
        rows = _prefix_rows(lg, n)
        if rows is None:
            continue
        for counts in _matrices(rows, rg):
            out.append(("c", left, right, counts))
    return out


def cost_of(node: Node) -> int:
    """Summed rank of a tree's contraction results (the reference's tie-break)."""
    if node[0] == "b":
        return 0
    return cost_of(node[1]) + cost_of(node[2]) + rank_of(node)


# ---------------------------------------------------------------------------
# dense evaluation on test vectors (dedupe and checks)
# ---------------------------------------------------------------------------
class DenseEval:
    """Dense-tensor values of nodes for one set of neighbours: unit vectors u
    [J, 3] and radial values rb [mu, J] (any numbers: the functions are told
    apart by value, not used as a potential)."""

    def __init__(self, u: np.ndarray, rb: np.ndarray):
        self.u, self.rb = u, rb
        self.cache: Dict[Node, np.ndarray] = {}

    def value(self, node: Node) -> np.ndarray:
        hit = self.cache.get(node)
        if hit is not None:
            return hit
        if node[0] == "b":
            _, mu, nu = node
            t = self.rb[mu].copy()                       # [J]
            for _ in range(nu):
                t = t[..., None] * self.u.reshape((self.u.shape[0],) + (1,) * (t.ndim - 1) + (3,))
            v = t.sum(axis=0)
        else:
            _, left, right, counts = node
            lv, rv = self.value(left), self.value(right)
            rg = groups_of(right)
            starts = np.cumsum((0,) + rg)[:-1]
            used = [0] * len(rg)
            rax = []
            for row in counts:
                for j, k in enumerate(row):
                    for _ in range(k):
                        rax.append(int(starts[j]) + used[j])
                        used[j] += 1
            v = np.tensordot(lv, rv, axes=(list(range(len(rax))), rax))
        self.cache[node] = v
        return v


def test_inputs(mu_count: int, seed: int = 12345, neighbours: int = 7):
    """Random unit vectors and radial values that tell the basis functions apart."""
    rng = np.random.default_rng(seed)
    u = rng.normal(size=(neighbours, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    rb = rng.uniform(0.5, 1.5, size=(mu_count, neighbours))
    return u, rb


# ---------------------------------------------------------------------------
# enumeration
# ---------------------------------------------------------------------------
def _trees(moments: Sequence[Node]) -> List[Node]:
    """Contraction trees over the given basic moments (positions distinct),
    in the shapes the reference enumerates (moment_jax.py:244-333): a pair; a
    pair then the third moment on the left; for four, a pair, then on its left
    either a third moment (and the last one on the left of that) or a
    contraction of the other two."""
    k = len(moments)
    if k == 1:
        return [moments[0]]
    idx = range(k)
    firsts = []
    for i, j in itertools.combinations(idx, 2):
        for c in contractions(moments[i], moments[j]):
            firsts.append((c, (i, j)))
    if k == 2:
        return [c for c, _ in firsts]
    out = []
    for c1, used in firsts:
        rest = [i for i in idx if i not in used]
        if k == 3:
            out.extend(contractions(moments[rest[0]], c1))
            continue
        others = [(moments[i], (i,)) for i in rest]
        for a, b in itertools.combinations(rest, 2):
            others += [(c, (a, b)) for c in contractions(moments[a], moments[b])]
        for other, took in others:
            for c2 in contractions(other, c1):
                if len(took) == 2:
                    out.append(c2)
                else:
                    last = [i for i in rest if i not in took][0]
                    out.extend(contractions(moments[last], c2))
    return out


def enumerate_scalars(level: int, max_moments: Optional[int] = DEFAULT_MAX_MOMENTS,
                      rtol: float = 1e-8, mu_max: Optional[int] = None,
                      nu_max: Optional[int] = None) -> List[Node]:
    """The scalar basis functions of a level: for every multiset of basic
    moments within the level (mu <= (level - 2) / 4, nu <= level / 2 - 2, at
    most max_moments of them, moment_jax.py:175-199), one tree per distinct
    scalar value on the test vectors, the cheapest of its equals.  mu_max and
    nu_max lower those limits (MLIP's level-28 template keeps mu <= 5 and
    nu <= 10, the level-24 limits)."""
    mu_lim = (level - 2) // 4
    nu_lim = max(level // 2 - 2, 0)
    mu_max = mu_lim if mu_max is None else min(mu_lim, mu_max)
    nu_max = nu_lim if nu_max is None else min(nu_lim, nu_max)
    k_max = level // 2 if max_moments is None else min(level // 2, max_moments)
    u, rb = test_inputs(mu_max + 1)
    ev = DenseEval(u, rb)
    singles = [(mu, nu) for mu in range(mu_max + 1) for nu in range(nu_max + 1)]
    out: List[Node] = []
    for k in range(1, k_max + 1):
        for combo in itertools.combinations_with_replacement(singles, k):
            if sum(level_of(mu, nu) for mu, nu in combo) > level:
                continue
            moments = [("b", mu, nu) for mu, nu in combo]
            found: List[Tuple[float, Node]] = []
            for t in _trees(moments):
                if rank_of(t) != 0:
                    continue
                val = float(ev.value(t))
                for i, (v0, t0) in enumerate(found):
                    if abs(val - v0) <= rtol * abs(v0):
                        if cost_of(t) < cost_of(t0):
                            found[i] = (v0, t)
                        break
                else:
                    found.append((val, t))
            out.extend(t for _, t in found)
        ev.cache.clear()
    return out


# ---------------------------------------------------------------------------
# MLIP tables
# ---------------------------------------------------------------------------
Mono = Tuple[int, int, int]
Key = Tuple[Node, Tuple[Mono, ...]]      # a component: node and one monomial per axis group

MAX_MULT = (1 << 14) - 1                 # entries carry multiplicities below 2^14


def _compositions(n: int):
    """(x, y, z) counts of n axes and the number of index tuples with them."""
    for x in range(n + 1):
        for y in range(n - x + 1):
            z = n - x - y
            yield (x, y, z), math.factorial(n) // (math.factorial(x) * math.factorial(y) * math.factorial(z))


def _add(a: Mono, b: Mono) -> Mono:
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def expand(key: Key) -> Dict[Tuple[Key, Key], int]:
    """Products that make up one component of a contraction:
    {(left component, right component): multiplicity}.  The free axes of each
    operand group carry the component's monomial for that group; the
    contracted axes between left group g and right group h add the same
    monomial c_gh to both sides, taken multinomial(n_gh; c_gh) times."""
    node, label = key
    _, left, right, counts = node
    lg, rg = groups_of(left), groups_of(right)
    zero = (0, 0, 0)
    it = iter(label)
    free_l = [next(it) if g - sum(row) > 0 else zero for g, row in zip(lg, counts)]
    free_r = [next(it) if h - sum(counts[i][j] for i in range(len(lg))) > 0 else zero for j, h in enumerate(rg)]
    blocks = [(i, j, counts[i][j]) for i in range(len(lg)) for j in range(len(rg)) if counts[i][j] > 0]
    out: Dict[Tuple[Key, Key], int] = {}
    for choice in itertools.product(*[list(_compositions(n)) for _, _, n in blocks]):
        ml, mr, mult = list(free_l), list(free_r), 1
        for (i, j, _), (c, w) in zip(blocks, choice):
            ml[i] = _add(ml[i], c)
            mr[j] = _add(mr[j], c)
            mult *= w
        k = ((left, tuple(ml)), (right, tuple(mr)))
        out[k] = out.get(k, 0) + mult
    return out


@dataclass
class BasisTables:
    """MLIP tables of a basis: basic moments (mu, a, b, c), products
    (i1, i2, mult, i3) in evaluation order, the scalar outputs."""
    level: int
    radial_funcs_count: int
    basic: np.ndarray                     # [B, 4]
    times: np.ndarray                     # [T, 4]
    mapping: np.ndarray                   # [Sa]
    moments_count: int
    scalars: List[Node] = field(default_factory=list)


def compile_tables(level: int, scalars: Sequence[Node]) -> BasisTables:
    """MLIP tables for the given scalar trees: every component the scalars need
    (no more), basic moments first, then intermediates with each one's
    products after those of its operands."""
    exp: Dict[Key, Dict[Tuple[Key, Key], int]] = {}
    order: List[Key] = []                 # intermediates, operands first
    basic_keys: Dict[Key, None] = {}

    def visit(key: Key):
        if key[0][0] == "b":
            basic_keys.setdefault(key, None)
            return
        if key in exp:
            return
        parts = expand(key)
        exp[key] = parts
        for lk, rk in parts:
            visit(lk)
            visit(rk)
        order.append(key)

    out_keys = [(s, ()) for s in scalars]
    for k in out_keys:          # recursion depth: the tree depth (at most four moments)
        visit(k)
    # basic moments by (mu, degree, a, b), then every intermediate in order
    def mono_of(k: Key) -> Mono:
        return k[1][0] if k[1] else (0, 0, 0)
    bkeys = sorted(basic_keys, key=lambda k: (k[0][1], sum(mono_of(k)), mono_of(k)))
    index: Dict[Key, int] = {k: i for i, k in enumerate(bkeys)}
    for k in order:
        index[k] = len(index)
    basic = np.array([(k[0][1],) + mono_of(k) for k in bkeys], dtype=np.int64).reshape(-1, 4)
    times = []
    for k in order:
        merged: Dict[Tuple[int, int], int] = {}
        for (lk, rk), m in exp[k].items():
            a, b = sorted((index[lk], index[rk]))
            merged[(a, b)] = merged.get((a, b), 0) + m
        for (a, b), m in merged.items():
            while m > 0:                  # multiplicities above the entry field split
                part = min(m, MAX_MULT)
                times.append((a, b, part, index[k]))
                m -= part
    mapping = np.array([index[k] for k in out_keys], dtype=np.int64)
    return BasisTables(level=level, radial_funcs_count=(level - 2) // 4 + 1, basic=basic,
                       times=np.array(times, dtype=np.int64).reshape(-1, 4), mapping=mapping,
                       moments_count=len(index), scalars=list(scalars))


def build_basis(level: int, max_moments: Optional[int] = DEFAULT_MAX_MOMENTS, mu_max: Optional[int] = None,
                nu_max: Optional[int] = None) -> BasisTables:
    """Enumerate a level's scalar basis and compile it to MLIP tables."""
    if level < 2:
        raise ValueError("level must be at least 2")
    t = compile_tables(level, enumerate_scalars(level, max_moments, mu_max=mu_max, nu_max=nu_max))
    t.radial_funcs_count = int(t.basic[:, 0].max()) + 1 if len(t.basic) else 1
    return t


def table_values(tables: BasisTables, u: np.ndarray, rb: np.ndarray) -> np.ndarray:
    """The scalar functions of the tables on neighbours (u, rb), evaluated the
    way the MLIP tables define them (basic moments, then the products)."""
    m = np.zeros(tables.moments_count)
    for k, (mu, a, b, c) in enumerate(tables.basic):
        m[k] = (rb[mu] * u[:, 0] ** a * u[:, 1] ** b * u[:, 2] ** c).sum()
    for i1, i2, mult, i3 in tables.times:
        m[i3] += mult * m[i1] * m[i2]
    return m[tables.mapping]


def template_potential(level: int, species_count: int, radial_basis_size: int = 8,
                       min_dist: float = 2.0, max_dist: float = 5.0,
                       max_moments: Optional[int] = DEFAULT_MAX_MOMENTS, mu_max: Optional[int] = None,
                       nu_max: Optional[int] = None):
    """An untrained `.mtp` potential of a level (the role of the reference's
    untrained_mtps/<level>.mtp templates): the generated basis, zero
    coefficients.  Fill them with mtp_file.with_random_coeffs or by training."""
    from .mtp_file import MTPPotential
    t = build_basis(level, max_moments, mu_max=mu_max, nu_max=nu_max)
    S, R, K = int(species_count), t.radial_funcs_count, int(radial_basis_size)
    pot = MTPPotential(species_count=S, min_dist=float(min_dist), max_dist=float(max_dist),
                       radial_basis_size=K, radial_funcs_count=R,
                       radial_coeffs=np.zeros((S, S, R, K)), alpha_moments_count=t.moments_count,
                       alpha_index_basic_count=len(t.basic), alpha_index_basic=t.basic,
                       alpha_index_times_count=len(t.times), alpha_index_times=t.times,
                       alpha_scalar_moments=len(t.mapping), alpha_moment_mapping=t.mapping,
                       species_coeffs=np.zeros(S), moment_coeffs=np.zeros(len(t.mapping)))
    pot.potential_tag = f"level {level}, basis generated from the level"
    pot.validate()
    return pot


def mlip_values(pot, u: np.ndarray, rb: np.ndarray) -> np.ndarray:
    """The scalar basis functions of a potential's MLIP tables on neighbours
    (u, rb) (basic moments, then the products, conversion.py:39-84)."""
    basic = np.asarray(pot.alpha_index_basic).reshape(-1, 4)
    times = np.asarray(pot.alpha_index_times).reshape(-1, 4)
    m = np.zeros(pot.alpha_moments_count)
    for k, (mu, a, b, c) in enumerate(basic):
        m[k] = (rb[mu] * u[:, 0] ** a * u[:, 1] ** b * u[:, 2] ** c).sum()
    for i1, i2, mult, i3 in times:
        m[i3] += mult * m[i1] * m[i2]
    return m[np.asarray(pot.alpha_moment_mapping)]


def remap_moment_coeffs(src, dst, rtol: float = 1e-8, seed: int = 2024) -> np.ndarray:
    """The moment coefficients of potential src, ordered for the basis of
    potential dst: each basis function of dst is found among src's by its value
    on random neighbours (the reference's BasisConverter matches the same way,
    conversion.py:112-168).  Every function of either basis must have exactly
    one partner; otherwise ValueError."""
    R = max(int(np.max(np.asarray(src.alpha_index_basic)[:, 0])),
            int(np.max(np.asarray(dst.alpha_index_basic)[:, 0]))) + 1
    u, rb = test_inputs(R, seed=seed, neighbours=11)
    vs, vd = mlip_values(src, u, rb), mlip_values(dst, u, rb)
    if len(vs) != len(vd):
        raise ValueError(f"the bases differ in size: {len(vs)} and {len(vd)} functions")
    free = np.ones(len(vs), bool)
    out = np.empty(len(vd))
    for i, x in enumerate(vd):
        hit = np.flatnonzero(free & (np.abs(vs - x) <= rtol * abs(x)))
        if len(hit) == 0:
            raise ValueError(f"basis function {i} of the target has no partner in the source")
        free[hit[0]] = False
        out[i] = np.asarray(src.moment_coeffs)[hit[0]]
    return out


def main(argv=None) -> int:
    """python -m mtp_b200.basis LEVEL SPECIES OUT.mtp [options]: write an
    untrained potential of a level (zero coefficients)."""
    import argparse
    from .mtp_file import write_mtp
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("level", type=int)
    ap.add_argument("species", type=int)
    ap.add_argument("out")
    ap.add_argument("--radial-basis-size", type=int, default=8)
    ap.add_argument("--min-dist", type=float, default=2.0)
    ap.add_argument("--max-dist", type=float, default=5.0)
    ap.add_argument("--max-moments", type=int, default=DEFAULT_MAX_MOMENTS)
    ap.add_argument("--mu-max", type=int, default=None)
    ap.add_argument("--nu-max", type=int, default=None)
    a = ap.parse_args(argv)
    pot = template_potential(a.level, a.species, a.radial_basis_size, a.min_dist, a.max_dist, a.max_moments,
                             a.mu_max, a.nu_max)
    write_mtp(a.out, pot)
    print(f"level {a.level}: {pot.alpha_scalar_moments} basis functions, {pot.alpha_moments_count} moments, "
          f"{pot.alpha_index_basic_count} basic, {pot.alpha_index_times_count} products -> {a.out}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
