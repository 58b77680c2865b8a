"""Reader and writer for MLIP ``.mtp`` potential files.

The format is the one the reference reads with ``read_mtp``
(motep_original_files/mtp.py:31-70) and writes with ``write_mtp``
(motep_original_files/mtp.py:93-139):

* a first line ``MTP``;
* ``key = value`` lines; scalars are ints or floats, lists are written
  ``{a, b, c}`` and tables ``{{...}, {...}}``;
* a ``radial_coeffs`` block holding, for every ordered species pair
  ``i-j`` (``i`` the centre species, ``j`` the neighbour species), a header
  line ``i-j`` followed by ``radial_funcs_count`` rows of
  ``radial_basis_size`` coefficients.

``alpha_index_basic`` rows are ``(mu, a, b, c)``: radial function ``mu``
times the monomial ``x^a y^b z^c`` of the neighbour unit vector.
``alpha_index_times`` rows are ``(i1, i2, mult, i3)``: moment ``i3`` gains
``mult * m[i1] * m[i2]``.  ``alpha_moment_mapping`` lists the moments that
form the scalar basis, one per entry of ``moment_coeffs``.
"""

from __future__ import annotations

import dataclasses
import io
import os
import re
from typing import Optional

import numpy as np

__all__ = ["MTPPotential", "MTPFormatError", "read_mtp", "write_mtp", "parse_mtp_text", "format_mtp",
           "with_random_coeffs"]


class MTPFormatError(ValueError):
    """Raised for a malformed ``.mtp`` file."""


@dataclasses.dataclass
class MTPPotential:
    """All fields of an ``.mtp`` file (names as in the file)."""

    version: str = "1.1.0"
    potential_name: str = "MTP1m"
    scaling: float = 1.0
    species_count: int = 0
    potential_tag: str = ""
    radial_basis_type: str = "RBChebyshev"
    min_dist: float = float("nan")
    max_dist: float = float("nan")
    radial_basis_size: int = 0
    radial_funcs_count: int = 0
    radial_coeffs: Optional[np.ndarray] = None  # [S, S, R, K] float64
    alpha_moments_count: int = 0
    alpha_index_basic_count: int = 0
    alpha_index_basic: Optional[np.ndarray] = None  # [B, 4] int64
    alpha_index_times_count: int = 0
    alpha_index_times: Optional[np.ndarray] = None  # [T, 4] int64
    alpha_scalar_moments: int = 0
    alpha_moment_mapping: Optional[np.ndarray] = None  # [Sa] int64
    species_coeffs: Optional[np.ndarray] = None  # [S] float64
    moment_coeffs: Optional[np.ndarray] = None  # [Sa] float64

    # ------------------------------------------------------------------
    def copy(self) -> "MTPPotential":
        out = dataclasses.replace(self)
        for f in dataclasses.fields(self):
            v = getattr(self, f.name)
            if isinstance(v, np.ndarray):
                setattr(out, f.name, v.copy())
        return out

    def validate(self, require_coeffs: bool = True) -> None:
        """Check the internal consistency of the tables (raises MTPFormatError).

        ``require_coeffs=False`` accepts an untrained template, which carries
        the basis tables but no coefficients.
        """
        S, R, K = self.species_count, self.radial_funcs_count, self.radial_basis_size
        if S <= 0 or R <= 0 or K <= 0:
            raise MTPFormatError("species_count, radial_funcs_count and radial_basis_size must be positive")
        if require_coeffs and (self.radial_coeffs is None or self.radial_coeffs.shape != (S, S, R, K)):
            raise MTPFormatError(f"radial_coeffs must have shape {(S, S, R, K)}")
        M = self.alpha_moments_count
        B = self.alpha_index_basic.shape[0]
        if B != self.alpha_index_basic_count:
            raise MTPFormatError("alpha_index_basic_count does not match the table")
        if self.alpha_index_times.shape[0] != self.alpha_index_times_count:
            raise MTPFormatError("alpha_index_times_count does not match the table")
        if len(self.alpha_moment_mapping) != self.alpha_scalar_moments:
            raise MTPFormatError("alpha_scalar_moments does not match alpha_moment_mapping")
        if require_coeffs:
            if self.moment_coeffs is None or len(self.moment_coeffs) != self.alpha_scalar_moments:
                raise MTPFormatError("moment_coeffs must have alpha_scalar_moments entries")
            if self.species_coeffs is None or len(self.species_coeffs) != S:
                raise MTPFormatError("species_coeffs must have species_count entries")
        if B > M:
            raise MTPFormatError("more basic moments than moments")
        if B and (self.alpha_index_basic[:, 0].max() >= R or self.alpha_index_basic.min() < 0):
            raise MTPFormatError("alpha_index_basic refers to a radial function >= radial_funcs_count")
        t = self.alpha_index_times
        if len(t) and (t[:, [0, 1, 3]].min() < 0 or t[:, [0, 1, 3]].max() >= M):
            raise MTPFormatError("alpha_index_times refers to a moment out of range")
        mp = self.alpha_moment_mapping
        if len(mp) and (mp.min() < 0 or mp.max() >= M):
            raise MTPFormatError("alpha_moment_mapping refers to a moment out of range")

    # ------------------------------------------------------------------
    @property
    def max_degree(self) -> int:
        b = self.alpha_index_basic
        return int(b[:, 1:].sum(axis=1).max()) if len(b) else 0


_INT_KEYS = {
    "species_count", "radial_basis_size", "radial_funcs_count", "alpha_moments_count",
    "alpha_index_basic_count", "alpha_index_times_count", "alpha_scalar_moments",
}
_FLOAT_KEYS = {"scaling", "min_dist", "max_dist"}
_TABLE_KEYS = {"alpha_index_basic", "alpha_index_times"}
_FLOAT_LIST_KEYS = {"species_coeffs", "moment_coeffs"}


def _parse_list(text: str, dtype) -> np.ndarray:
    body = text.strip()
    if not (body.startswith("{") and body.endswith("}")):
        raise MTPFormatError(f"expected a {{...}} list, got {body[:40]!r}")
    body = body[1:-1].strip()
    if not body:
        return np.zeros(0, dtype=dtype)
    try:
        return np.array([dtype(tok) for tok in body.split(",")], dtype=dtype)
    except ValueError as exc:
        raise MTPFormatError(f"bad list entry: {exc}") from None


def _parse_table(text: str) -> np.ndarray:
    body = text.strip()
    if not (body.startswith("{") and body.endswith("}")):
        raise MTPFormatError("expected a {{...}} table")
    rows = re.findall(r"\{([^{}]*)\}", body[1:-1])
    if not rows:
        return np.zeros((0, 4), dtype=np.int64)
    out = []
    for r in rows:
        vals = [int(tok) for tok in r.split(",") if tok.strip()]
        if len(vals) != 4:
            raise MTPFormatError(f"table rows must have 4 entries, got {r!r}")
        out.append(vals)
    return np.array(out, dtype=np.int64)


def parse_mtp_text(text: str, require_coeffs: bool = True) -> MTPPotential:
    """Parse the contents of an ``.mtp`` file (``require_coeffs=False`` for a template)."""
    lines = text.splitlines()
    pot = MTPPotential()
    fields = {}
    i = 0
    saw_header = False
    while i < len(lines):
        line = lines[i].strip()
        i += 1
        if not line:
            continue
        if line == "MTP":
            saw_header = True
            continue
        if line == "radial_coeffs":
            S = fields.get("species_count")
            R = fields.get("radial_funcs_count")
            K = fields.get("radial_basis_size")
            if S is None or R is None or K is None:
                raise MTPFormatError("radial_coeffs before species_count/radial_funcs_count/radial_basis_size")
            rc = np.full((S, S, R, K), np.nan)
            for _ in range(S * S):
                if i >= len(lines):
                    raise MTPFormatError("truncated radial_coeffs block")
                hdr = lines[i].strip()
                i += 1
                m = re.fullmatch(r"(\d+)\s*-\s*(\d+)", hdr)
                if not m:
                    raise MTPFormatError(f"expected 'i-j' species pair, got {hdr!r}")
                a, b = int(m.group(1)), int(m.group(2))
                if a >= S or b >= S:
                    raise MTPFormatError(f"species pair {hdr} out of range")
                for mu in range(R):
                    if i >= len(lines):
                        raise MTPFormatError("truncated radial_coeffs block")
                    row = _parse_list(lines[i], float)
                    i += 1
                    if len(row) != K:
                        raise MTPFormatError(f"radial_coeffs row has {len(row)} entries, expected {K}")
                    rc[a, b, mu] = row
            if np.isnan(rc).any():
                raise MTPFormatError("radial_coeffs block does not cover every species pair")
            fields["radial_coeffs"] = rc
            continue
        if "=" not in line:
            raise MTPFormatError(f"unrecognised line {line!r}")
        key, value = (s.strip() for s in line.split("=", 1))
        try:
            if key in _INT_KEYS:
                fields[key] = int(value)
            elif key in _FLOAT_KEYS:
                fields[key] = float(value)
            elif key in _TABLE_KEYS:
                fields[key] = _parse_table(value)
            elif key == "alpha_moment_mapping":
                fields[key] = _parse_list(value, int).astype(np.int64)
            elif key in _FLOAT_LIST_KEYS:
                fields[key] = _parse_list(value, float)
            else:
                fields[key] = value
        except ValueError as exc:
            raise MTPFormatError(f"bad value for {key}: {exc}") from None
    if not saw_header:
        raise MTPFormatError("missing 'MTP' header line")
    known = {f.name for f in dataclasses.fields(MTPPotential)}
    for k, v in fields.items():
        if k in known:
            setattr(pot, k, v)
    for k in ("alpha_index_basic", "alpha_index_times"):
        if getattr(pot, k) is None:
            setattr(pot, k, np.zeros((0, 4), dtype=np.int64))
    if pot.alpha_moment_mapping is None:
        pot.alpha_moment_mapping = np.zeros(0, dtype=np.int64)
    pot.validate(require_coeffs)
    return pot


def read_mtp(path: os.PathLike, require_coeffs: bool = True) -> MTPPotential:
    with open(path, "r", encoding="utf-8") as fh:
        return parse_mtp_text(fh.read(), require_coeffs)


def _fmt_float(v: float) -> str:
    # 17 significant digits: the file round-trips every double exactly.
    return f"{float(v):.16e}"


def _fmt_list(vals, fmt) -> str:
    return "{" + ", ".join(fmt(v) for v in vals) + "}"


def format_mtp(pot: MTPPotential) -> str:
    pot.validate()
    out = io.StringIO()
    w = out.write
    w("MTP\n")
    w(f"version = {pot.version}\n")
    w(f"potential_name = {pot.potential_name}\n")
    w(f"scaling = {_fmt_float(pot.scaling)}\n")
    w(f"species_count = {pot.species_count:d}\n")
    w(f"potential_tag = {pot.potential_tag}\n")
    w(f"radial_basis_type = {pot.radial_basis_type}\n")
    w(f"\tmin_dist = {_fmt_float(pot.min_dist)}\n")
    w(f"\tmax_dist = {_fmt_float(pot.max_dist)}\n")
    w(f"\tradial_basis_size = {pot.radial_basis_size:d}\n")
    w(f"\tradial_funcs_count = {pot.radial_funcs_count:d}\n")
    w("\tradial_coeffs\n")
    S = pot.species_count
    for a in range(S):
        for b in range(S):
            w(f"\t\t{a}-{b}\n")
            for row in pot.radial_coeffs[a, b]:
                w("\t\t\t" + _fmt_list(row, _fmt_float) + "\n")
    w(f"alpha_moments_count = {pot.alpha_moments_count:d}\n")
    w(f"alpha_index_basic_count = {pot.alpha_index_basic_count:d}\n")
    w("alpha_index_basic = {" + ", ".join(_fmt_list(r, str) for r in pot.alpha_index_basic.tolist()) + "}\n")
    w(f"alpha_index_times_count = {pot.alpha_index_times_count:d}\n")
    w("alpha_index_times = {" + ", ".join(_fmt_list(r, str) for r in pot.alpha_index_times.tolist()) + "}\n")
    w(f"alpha_scalar_moments = {pot.alpha_scalar_moments:d}\n")
    w("alpha_moment_mapping = " + _fmt_list(pot.alpha_moment_mapping.tolist(), str) + "\n")
    w("species_coeffs = " + _fmt_list(pot.species_coeffs, _fmt_float) + "\n")
    w("moment_coeffs = " + _fmt_list(pot.moment_coeffs, _fmt_float) + "\n")
    return out.getvalue()


def write_mtp(path: os.PathLike, pot: MTPPotential) -> None:
    with open(path, "w", encoding="utf-8") as fh:
        fh.write(format_mtp(pot))


def with_random_coeffs(template: MTPPotential, seed: int, species_count: Optional[int] = None,
                       radial_funcs_count: Optional[int] = None, min_dist: Optional[float] = None,
                       max_dist: Optional[float] = None, scaling: float = 1.0,
                       radial_sigma: float = 0.1, basis_sigma: float = 0.01,
                       species_shift: float = -3.0) -> MTPPotential:
    """A potential with the template's basis tables and seeded random coefficients.

    Draw order with ``numpy.random.default_rng(seed)``: radial coefficients
    ``[S, S, R, K] ~ N(0, radial_sigma^2)`` first, then moment (basis)
    coefficients ``[Sa] ~ N(0, basis_sigma^2)``.  Species coefficients are
    all ``species_shift``.
    """
    pot = template.copy()
    if species_count is not None:
        pot.species_count = int(species_count)
    if radial_funcs_count is not None:
        need = int(pot.alpha_index_basic[:, 0].max()) + 1 if len(pot.alpha_index_basic) else 1
        if radial_funcs_count < need:
            raise MTPFormatError(f"the basis needs radial_funcs_count >= {need}")
        pot.radial_funcs_count = int(radial_funcs_count)
    if min_dist is not None:
        pot.min_dist = float(min_dist)
    if max_dist is not None:
        pot.max_dist = float(max_dist)
    pot.scaling = float(scaling)
    rng = np.random.default_rng(seed)
    S, R, K = pot.species_count, pot.radial_funcs_count, pot.radial_basis_size
    pot.radial_coeffs = rng.normal(0.0, radial_sigma, size=(S, S, R, K))
    pot.moment_coeffs = rng.normal(0.0, basis_sigma, size=pot.alpha_scalar_moments)
    pot.species_coeffs = np.full(S, float(species_shift))
    pot.validate()
    return pot
