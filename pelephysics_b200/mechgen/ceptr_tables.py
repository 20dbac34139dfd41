"""Mechanism front-end: Cantera-style YAML -> flat C tables for the engine.

The reference turns a mechanism into straight-line C++ with its CEPTR
generator (Support/ceptr/ceptr/*.py, which needs Cantera).  This module reads
the same ``mechanism.yaml`` with PyYAML and produces *data tables* instead of
code: every number the generated ``mechanism.H`` would hard-wire is computed
with the same formula and rounded through the same printf format, so that a
table-driven evaluator reproduces the reference's arithmetic.  The conventions
reproduced, with the reference lines they follow:

* reaction order: Troe, SRI, Lindemann fall-off, then third-body (including an
  explicit collider), then elementary (Support/ceptr/ceptr/reaction_info.py:36-130)
* an elementary reaction with one species on both sides and three molecules
  on either side is a three-body reaction with that species as sole collider
  (the Cantera 3 parse the reference mechanisms were generated with; e.g.
  Mechanisms/drm19/mechanism.H "reaction 17: H + O2 + O2 <=> HO2 + O2")
* SI pre-exponential ``%.15g`` (production.py:1130-1170), Ea/R in K with
  Rc = 1.98721558317399615845 cal/mol/K (constants.py:11), fall-off low-pressure
  factor ``10**(-6 dim) * low_pef * 10**3**dim`` (production.py:1216-1222) and
  the Jacobian's ``k_0 = low_pef * 10**3**dim`` (jacobian.py:826-858)
* efficiencies as ``mixture + sum (eff-1) c`` with ``(eff-1)`` printed ``%.15g``
  (production.py:1504-1582) and ``eff`` printed ``%.15g`` for the Jacobian
  (utilities.py:391-453, jacobian.py:1365-1395)
* Troe coefficients as printed by production.py:1226-1268 and
  jacobian.py:885-940
* refC power of the reverse rate, including the dropped conversion for a
  change of moles <= -2 (utilities.py:183-281)
* NASA-7 coefficient sets per thermo routine with the routine's own format
  (thermo.py:501-694): ``+15.8e`` for cv, cp, e, h, dcp/dT; ``+20.15e`` for g;
  a species whose two ranges agree under ``np.allclose(atol=1e-22)`` keeps only
  its high range (thermo.py:234-261)
* molecular weights ``%f`` and inverse weights ``%.16f`` (ck.py, thermo.py:395)

Run as ``python -m pelephysics_b200.mechgen.ceptr_tables <reference-root>``;
it writes ``pelephysics_b200/csrc/mech/mech_<name>.h`` for the four
mechanisms the engine ships with.
"""

from __future__ import annotations

import os
import re
import sys
from collections import Counter, OrderedDict

import numpy as np
import yaml

MECHS = ["LiDryer", "drm19", "dodecane_lu", "heptane_lu_88sk", "CH4_lean_qss", "C1-C2-NO_qss", "LuEthylene_qss",
         "grimech30", "FFCM1_Red", "chem-H"]

RC = 1.98721558317399615845  # cal/mol/K
ATOMIC_WEIGHTS = {
    "H": 1.008,
    "He": 4.002602,
    "C": 12.011,
    "N": 14.007,
    "O": 15.999,
    "Ar": 39.95,
}

# table widths (checked by assertions below)
MAXPS = 6  # phase-space entries (species, order) per side
MAXW = 8  # production-rate wdot updates per reaction
MAXKC = 10  # Gibbs terms of the equilibrium exponent
MAXJN = 8  # Jacobian net-stoichiometry entries

K_SIMPLE, K_THIRD, K_COLLIDER, K_TROE, K_LINDEMANN, K_SRI = range(6)


class _Yaml12Loader(yaml.SafeLoader):
    """PyYAML's safe loader with YAML 1.2 booleans (true / false only), as
    Cantera reads its files: a species named NO (nitric oxide) stays a
    string instead of YAML 1.1's False."""


for _ch, _res in list(_Yaml12Loader.yaml_implicit_resolvers.items()):
    _Yaml12Loader.yaml_implicit_resolvers[_ch] = [(t, r) for t, r in _res if t != "tag:yaml.org,2002:bool"]
_Yaml12Loader.add_implicit_resolver("tag:yaml.org,2002:bool", re.compile(r"^(?:true|True|TRUE|false|False|FALSE)$"),
                                    list("tTfF"))


def load_yaml(path):
    with open(path) as fh:
        return yaml.load(fh, Loader=_Yaml12Loader)


def fmt(x: float, f: str) -> float:
    """Round ``x`` through a printf format, as the generated source does."""
    return float(format(x, f))


def _parse_side(s: str):
    s = s.strip()
    fall = None
    m = re.search(r"\(\+\s*([^)]+)\)\s*$", s)
    if m:
        fall = m.group(1).strip()
        s = s[: m.start()].strip()
    toks = [t.strip() for t in re.split(r"\s\+\s", " " + s + " ") if t.strip()]
    side = OrderedDict()
    has_m = False
    for t in toks:
        mm = re.match(r"^(\d+(?:\.\d+)?)\s+(\S+)$", t)
        if mm:
            nu, sp = float(mm.group(1)), mm.group(2)
        else:
            nu, sp = 1.0, t
        if sp == "M":
            has_m = True
            continue
        side[sp] = side.get(sp, 0.0) + nu
    return side, has_m, fall


def parse_equation(eq: str):
    if "<=>" in eq:
        lhs, rhs = eq.split("<=>")
        rev = True
    elif "=>" in eq:
        lhs, rhs = eq.split("=>")
        rev = False
    else:
        lhs, rhs = eq.split("=")
        rev = True
    r, rm, rf = _parse_side(lhs)
    p, pm, pf = _parse_side(rhs)
    return r, p, (rm or pm), (rf or pf), rev


class Reaction:
    """One reaction in the form the CEPTR generator sees it."""

    def __init__(self, idx, d, species):
        self.orig = idx
        self.eq = d["equation"]
        r, p, has_m, fall, rev = parse_equation(self.eq)
        self.reversible = bool(rev) and d.get("reversible", True) is not False
        rtype = d.get("type", "elementary")
        self.reactants = OrderedDict(r)
        self.products = OrderedDict(p)
        self.third = None  # dict of efficiencies
        self.default_eff = 1.0
        self.falloff = None
        if "orders" in d:
            raise NotImplementedError("explicit reaction orders")
        if d.get("negative-A") or "reverse" in d:
            raise NotImplementedError("negative-A / explicit reverse rate")
        if rtype == "three-body":
            self.third = {k: float(v) for k, v in d.get("efficiencies", {}).items()}
            self.default_eff = float(d.get("default-efficiency", 1.0))
            self.rate = d["rate-constant"]
        elif rtype == "falloff":
            if fall != "M":
                raise NotImplementedError("fall-off with a named collider")
            self.third = {k: float(v) for k, v in d.get("efficiencies", {}).items()}
            self.default_eff = float(d.get("default-efficiency", 1.0))
            self.rate = d["high-P-rate-constant"]
            self.low = d["low-P-rate-constant"]
            if "Troe" in d:
                t = d["Troe"]
                self.falloff = "Troe"
                self.troe = [float(t["A"]), float(t["T3"]), float(t["T1"])]
                if "T2" in t:
                    self.troe.append(float(t["T2"]))
            elif "SRI" in d:
                # The reference generator emits unbalanced parentheses for SRI
                # (production.py:1269-1300) and has no SRI Jacobian
                # (jacobian.py:878-880), so no reference mechanism uses it.
                raise NotImplementedError("SRI fall-off")
            else:
                self.falloff = "Lindemann"
        elif rtype == "elementary":
            self.rate = d["rate-constant"]
            both = [s for s in self.reactants if s in self.products]
            nr = sum(self.reactants.values())
            np_ = sum(self.products.values())
            if len(both) == 1 and max(nr, np_) >= 3:
                x = both[0]
                self.reactants[x] -= 1.0
                self.products[x] -= 1.0
                if self.reactants[x] == 0:
                    del self.reactants[x]
                if self.products[x] == 0:
                    del self.products[x]
                self.third = {x: 1.0}
                self.default_eff = 0.0
        else:
            raise NotImplementedError(f"reaction type {rtype}")
        for s in list(self.reactants) + list(self.products) + list(self.third or {}):
            if s not in species:
                raise KeyError(f"unknown species {s} in {self.eq}")

    @property
    def is_collider(self):
        return (
            self.third is not None
            and self.falloff is None
            and len(self.third) == 1
            and abs(self.default_eff) < 1e-9
        )

    @property
    def kind(self):
        if self.falloff == "Troe":
            return K_TROE
        if self.falloff == "Sri":
            return K_SRI
        if self.falloff == "Lindemann":
            return K_LINDEMANN
        if self.third is not None:
            return K_COLLIDER if self.is_collider else K_THIRD
        return K_SIMPLE


def ceptr_sort(reactions):
    """reaction_info.py:36-130: Troe, SRI, Lindemann, third-body, rest."""
    out = []
    for key in (
        lambda r: r.falloff == "Troe",
        lambda r: r.falloff == "Sri",
        lambda r: r.falloff == "Lindemann",
        lambda r: r.third is not None,
        lambda r: True,
    ):
        for r in reactions:
            if r not in out and key(r):
                out.append(r)
    return out


def species_weight(comp):
    return sum(ATOMIC_WEIGHTS[e] * n for e, n in comp.items())


def thermo_sets(coeffs):
    """Per-routine coefficient sets (thermo.py:501-694) for one NASA-7 range."""
    a = [float(c) for c in coeffs]
    f8 = lambda x: fmt(x, "+15.8e")
    f15 = lambda x: fmt(x, "+20.15e")
    return {
        "cv": [f8(a[0] - 1.0), f8(a[1]), f8(a[2]), f8(a[3]), f8(a[4])],
        "cp": [f8(a[0]), f8(a[1]), f8(a[2]), f8(a[3]), f8(a[4])],
        "dcp": [f8(a[1]), f8(a[2] * 2.0), f8(a[3] * 3.0), f8(a[4] * 4.0)],
        "u": [f8(a[0] - 1.0), f8(a[1] / 2), f8(a[2] / 3), f8(a[3] / 4), f8(a[4] / 5), f8(a[5])],
        "h": [f8(a[0]), f8(a[1] / 2), f8(a[2] / 3), f8(a[3] / 4), f8(a[4] / 5), f8(a[5])],
        # g/RT: invT, const, logT, T, T2, T3, T4
        "g": [
            f15(a[5]),
            f15(a[0] - a[6]),
            f15(-a[0]),
            f15(-a[1] / 2),
            f15(-a[2] / 6),
            f15(-a[3] / 12),
            f15(-a[4] / 20),
        ],
    }


def sorted_by_species(d, idx):
    return sorted(d.items(), key=lambda kv: idx[kv[0]])


def mechanism_file(mech_dir):
    """The mechanism's YAML: mechanism.yaml, or for a QSS mechanism of the
    reference (CEPTR's QSSA input) qssa.yaml, whose phase lists the species
    in steady state under ``qssa_species``."""
    for f in ("mechanism.yaml", "qssa.yaml"):
        path = os.path.join(mech_dir, f)
        if os.path.exists(path):
            return path
    raise FileNotFoundError(f"no mechanism.yaml or qssa.yaml in {mech_dir}")


def build(mech_dir, name):
    y = load_yaml(mechanism_file(mech_dir))
    # rate units: the Chemkin-converted mechanisms declare cm / mol / cal/mol;
    # a file without a units entry (Cantera's writer, e.g. qssa.yaml) is in
    # Cantera's own m / kmol / J/kmol, the units CEPTR converts from
    units = y.get("units", {})
    si_kmol = units.get("length", "m") == "m" and units.get("quantity", "kmol") == "kmol"
    if si_kmol:
        assert units.get("activation-energy", "J/kmol") == "J/kmol", units
    else:
        assert (units.get("length"), units.get("quantity"), units.get("activation-energy")) == (
            "cm", "mol", "cal/mol"), units
    phase = y["phases"][0]
    all_species = list(phase["species"])
    qss_set = set(phase.get("qssa_species", []))
    # transported species keep the mechanism's order; the QSS species (in the
    # mechanism's order too) take the slots after the unit slot nsp
    species = [s for s in all_species if s not in qss_set]
    qss = [s for s in all_species if s in qss_set]
    nsp = len(species)
    idx = {s: i for i, s in enumerate(species)}
    idx.update({s: nsp + 1 + q for q, s in enumerate(qss)})
    spdata = {s["name"]: s for s in y["species"]}
    # reactions whose forward rate the QSS reduction removes (their forward
    # would be quadratic in QSS species): productionRate uses qdot = -q_r
    rm_fwd = set(int(i) for i in phase.get("forward_to_remove_idx", []))
    nonq = os.path.join(mech_dir, "non_qssa_list.yaml")
    if qss and os.path.exists(nonq):
        listed = load_yaml(nonq)["species"]
        assert listed == species, (listed, species)

    # --- species data (mw, imw: transported species; thermo: transported,
    # then for a QSS mechanism an empty entry for the unit slot and the QSS
    # species, so that thermo entry == concentration slot)
    mw, imw, tmid, tlo, thi = [], [], [], [], []
    sets_lo, sets_hi = [], []
    thermo_species = species + ([None] + qss if qss else [])
    for s in thermo_species:
        if s is None:
            zero = {k: [0.0] * len(v) for k, v in thermo_sets([0.0] * 7).items()}
            tmid.append(None)
            tlo.append(0.0)
            thi.append(0.0)
            sets_lo.append(zero)
            sets_hi.append(zero)
            continue
        d = spdata[s]
        if s in idx and idx[s] < nsp:
            w = species_weight(d["composition"])
            mw.append(fmt(w, "f"))
            imw.append(fmt(1.0 / w, ".16f"))
        th = d["thermo"]
        assert th["model"] == "NASA7", th["model"]
        rng = th["temperature-ranges"]
        data = th["data"]
        if len(data) == 1:
            lo = hi = data[0]
            tm = None
        else:
            assert len(data) == 2
            lo, hi = data
            tm = float(rng[1])
            if np.allclose(np.array(hi, float), np.array(lo, float), atol=1e-22):
                lo = hi
                tm = None
        tmid.append(tm)
        tlo.append(float(rng[0]))
        thi.append(float(rng[-1]))
        sets_lo.append(thermo_sets(lo))
        sets_hi.append(thermo_sets(hi))

    # --- reactions
    rxns = [Reaction(i, d, idx) for i, d in enumerate(y["reactions"])]
    order = ceptr_sort(rxns)
    R = []
    for r in order:
        rec = {"orig": r.orig, "eq": r.eq, "kind": r.kind, "rev": int(r.reversible), "rmf": int(r.orig in rm_fwd)}
        # forward / reverse phase space (utilities.py:23-157): reactants plus
        # the explicit collider, sorted by species index
        fwd = Counter(r.reactants)
        rev = Counter(r.products)
        if r.is_collider:
            fwd = fwd + Counter(r.third)
            rev = rev + Counter(r.third)
        rec["fps"] = [(idx[s], float(v)) for s, v in sorted_by_species(dict(fwd), idx)]
        rec["rps"] = [(idx[s], float(v)) for s, v in sorted_by_species(dict(rev), idx)]
        assert len(rec["fps"]) <= MAXPS and len(rec["rps"]) <= MAXPS, r.eq
        for _, v in rec["fps"] + rec["rps"]:
            assert float(v).is_integer(), r.eq
        # dimension of the forward phase space (production.py:1118-1121)
        dim = sum(r.reactants.values())
        A = float(r.rate["A"])
        beta = float(r.rate["b"])
        Ea = float(r.rate["Ea"])
        if si_kmol:
            # Cantera's values as they are: k in (m^3/kmol)^(order-1)/s to
            # (m^3/mol)^(order-1)/s, Ea from J/kmol to cal/mol
            korder = dim + 1 if r.kind in (K_THIRD, K_COLLIDER) else dim
            pef = A * 1000.0 ** (1 - korder)
            Ea = Ea / 4184.0
        elif r.kind in (K_SIMPLE,):
            pef = A * 1e-6 ** (dim - 1)
        elif r.kind in (K_THIRD, K_COLLIDER):
            pef = A * 1e-6 ** dim
        else:
            pef = A * 1e-6 ** (dim - 1)
        rec["A"] = fmt(pef, ".15g")
        rec["beta"] = fmt(beta, ".15g")
        rec["EaR"] = fmt(Ea / RC, ".15g")
        if r.falloff is not None:
            L = r.low
            A0 = float(L["A"])
            # Cantera keeps the low-pressure factor in kmol units with one
            # more order than k_inf; CEPTR converts it with the k_inf factor
            # and rescales by 10**(-6 dim) * 10**(3**dim).
            A0_cantera = A0 if si_kmol else A0 * 1e-3 ** dim
            low_pef = A0_cantera * 1000.0 ** (1 - dim)
            rec["P0"] = fmt(10 ** (-dim * 6) * low_pef * 10 ** 3 ** dim, ".15g")
            rec["k0"] = fmt(low_pef * 10 ** 3 ** dim, ".15g")
            rec["beta0"] = fmt(float(L["b"]), ".15g")
            Ea0 = float(L["Ea"]) / 4184.0 if si_kmol else float(L["Ea"])
            rec["EaR0"] = fmt(Ea0 / RC, ".15g")
            rec["prdim"] = float(f"1e-{int(dim * 6)}")
            if r.falloff == "Troe":
                t = r.troe
                rec["troe"] = {
                    "n": len(t),
                    "a": fmt(t[0], ".15g"),
                    "T3": fmt(t[1], ".15g"),
                    "T1": fmt(t[2], ".15g"),
                    "T2": fmt(t[3], ".15g") if len(t) == 4 else 0.0,
                    "oma": fmt(1.0 - t[0], ".15g"),
                    "iT3": fmt(1.0 / t[1], ".15g") if abs(t[1]) > 1e-100 else 0.0,
                    "iT1": fmt(1.0 / t[2], ".15g") if abs(t[2]) > 1e-100 else 0.0,
                    "p1": int(abs(t[1]) > 1e-100 and (1.0 - t[0]) != 0),
                    "p2": int(abs(t[2]) > 1e-100 and t[0] != 0),
                    "j1": int(abs(t[1]) > 1e-100),
                    "j2": int(abs(t[2]) > 1e-100),
                    "j3": int(len(t) == 4 and abs(t[3]) > 1e-100),
                }
            if r.falloff == "Sri":
                s = r.sri
                rec["sri"] = [fmt(v, ".15g") for v in s] + ([1.0, 0.0] if len(s) == 3 else [])
                rec["sri_n"] = len(s)
        # efficiencies (production.py:1504-1582; jacobian enhancement)
        eff = []
        if r.third and any(s_ in qss_set for s_ in r.third):
            raise NotImplementedError("a QSS species as third body")
        if r.kind in (K_THIRD, K_TROE, K_LINDEMANN, K_SRI):
            for s, e in sorted_by_species(r.third, idx):
                eff.append((idx[s], fmt(e, ".15g"), fmt(e - 1.0, ".15g")))
        rec["eff"] = eff
        # refC power multiplying the reverse rate (utilities.py:183-281)
        dnu = sum(r.products.values()) - sum(r.reactants.values())
        assert float(dnu).is_integer()
        dnu = int(dnu)
        rec["kcpow"] = dnu if dnu >= -1 else 0
        # Gibbs terms of the equilibrium exponent (utilities.py:293-388):
        # per species in index order, reactant term (+) then product term (-)
        terms = []
        for s in species + qss:
            if s in r.reactants:
                terms.append((idx[s], float(r.reactants[s])))
            if s in r.products:
                terms.append((idx[s], -float(r.products[s])))
        assert len(terms) <= MAXKC, r.eq
        rec["kc"] = terms
        # production-rate wdot updates (production.py:1390-1430): agents =
        # distinct (species, coef) pairs sorted by species; a reactant entry
        # then a product entry for each
        agents = sorted(
            set(list(r.reactants.items()) + list(r.products.items())),
            key=lambda v: idx[v[0]],
        )
        wup = []
        for s, c in agents:
            if s in qss_set:
                continue  # no rate for a species in steady state
            if s in r.reactants and r.reactants[s] == c:
                wup.append((idx[s], -float(c)))
            if s in r.products and r.products[s] == c:
                wup.append((idx[s], float(c)))
        assert len(wup) <= MAXW, r.eq
        rec["wup"] = wup
        # Jacobian net stoichiometry over rea/pro dicts including a collider
        # (jacobian.py:620-690)
        rea = dict(fwd) if r.is_collider else dict(r.reactants)
        pro = dict(rev) if r.is_collider else dict(r.products)
        jn = []
        for k, s in enumerate(species):  # transported species only
            if s in rea and s in pro:
                nu = pro[s] - rea[s]
            elif s in rea:
                nu = -rea[s]
            elif s in pro:
                nu = pro[s]
            else:
                continue
            jn.append((k, float(nu)))
        assert len(jn) <= MAXJN, r.eq
        rec["jn"] = jn
        rec["sum_nuk"] = float(sum(pro.values()) - sum(rea.values()))
        rec["hr"] = [(idx[s], float(v)) for s, v in sorted_by_species(rea, idx)]
        rec["hp"] = [(idx[s], float(v)) for s, v in sorted_by_species(pro, idx)]
        R.append(rec)

    qss_info = qss_structure(order, qss, qss_set, rm_fwd) if qss else None
    return {
        "name": name,
        "qss": qss,
        "qss_info": qss_info,
        "species": species,
        "mw": mw,
        "imw": imw,
        "tmid": tmid,
        "tlo": tlo,
        "thi": thi,
        "lo": sets_lo,
        "hi": sets_hi,
        "rxns": R,
    }


def qss_structure(order, qss, qss_set, rm_fwd=()):
    """The steady-state balance of each QSS species, as the reference's
    generated comp_qss_coeff / comp_sc_qss form it
    (Support/ceptr/ceptr/qssa_converter.py: qssa_coeff_functions,
    qssa_component_functions): the reactions that involve a QSS species
    (in evaluation order, k = 0 ..) give coefficients q_f,k and q_r,k, the
    rates with the QSS concentrations left out.  For QSS species i, in k
    order, each direction of a reaction adds nu times its coefficient: to
    the loss (role -2) when it consumes i, to the production (role -1) when
    it makes i from transported species only, to the coupling with QSS
    species j (role j) when it makes i from j.  A direction that consumes
    more than one QSS molecule would make the balance nonlinear: the
    reference's reduction removes such a forward rate (forward_to_remove_idx
    of the mechanism's phase; its q_f is 0 in productionRate too, qdot = -q_r)
    and rejects any other, and so does this generator."""
    q_rx, terms = [], [[] for _ in qss]
    qi = {s: q for q, s in enumerate(qss)}
    for pos, r in enumerate(order):
        rq = [(s, float(v)) for s, v in r.reactants.items() if s in qss_set]
        pq = [(s, float(v)) for s, v in r.products.items() if s in qss_set]
        if not rq and not pq:
            continue
        k = len(q_rx)
        q_rx.append(pos)
        dirs = []
        if r.orig not in rm_fwd:
            dirs.append((2 * k, rq, pq))  # forward: consumes rq, makes pq
        if r.reversible:
            dirs.append((2 * k + 1, pq, rq))  # reverse: consumes pq, makes rq
        for term, cons, made in dirs:
            if len(cons) > 1 or any(v != 1.0 for _, v in cons):
                raise NotImplementedError(f"nonlinear QSS reaction {r.eq}")
            if cons and any(s == cons[0][0] for s, _ in made):
                raise NotImplementedError(f"QSS species on both sides of {r.eq}")
            if len(made) > 1:
                # a direction making two QSS species: the reverse of a
                # reaction whose forward is removed counts for each; an
                # irreversible forward the reference's converter leaves out
                # of every balance ("does not contribute to any QSSA
                # coefficients and is thus ignored"); from a QSS species, it
                # handles neither
                if cons:
                    raise NotImplementedError(f"QSS reaction {r.eq} turns a QSS species into two")
                if term % 2 == 0 and not r.reversible:
                    continue
            for s, v in cons:
                terms[qi[s]].append((term, -2, v))
            for s, v in made:
                terms[qi[s]].append((term, qi[cons[0][0]] if cons else -1, v))
    for q, lst in enumerate(terms):
        lst.sort(key=lambda t: t[0] // 2)  # k order (stable: a reaction's terms keep their order)
    off, term, role, coef = [0], [], [], []
    for lst in terms:
        for t, ro, v in lst:
            term.append(t)
            role.append(ro)
            coef.append(v)
        off.append(len(term))
    for q, lst in enumerate(terms):
        if not any(ro == -2 for _, ro, _ in lst) or not any(ro != -2 for _, ro, _ in lst):
            raise ValueError(f"QSS species {qss[q]} is not both produced and consumed")
    return {"q_rx": q_rx, "q_off": off, "q_term": term, "q_role": role, "q_coef": coef}


def _carr(ctype, name, vals, per_line=4):
    def f(v):
        if ctype == "double":
            return repr(float(v)) if np.isfinite(v) else "0.0"
        return str(int(v))

    body = ",\n  ".join(
        ", ".join(f(v) for v in vals[i : i + per_line]) for i in range(0, max(len(vals), 1), per_line)
    )
    if not vals:
        body = "0"
    return f"static const {ctype} {name}[] = {{\n  {body}\n}};\n"


def emit_header(M, path):
    name = M["name"]
    cid = re.sub(r"[^A-Za-z0-9_]", "_", name)  # C identifier (C1-C2-NO_qss -> C1_C2_NO_qss)
    nsp = len(M["species"])
    nr = len(M["rxns"])
    P = f"ppbm_{cid}_"
    out = []
    out.append(f"// Generated by pelephysics_b200/mechgen/ceptr_tables.py from\n")
    src = "qssa.yaml" if M["qss"] else "mechanism.yaml"
    out.append(f"// Mechanisms/{name}/{src} of the reference. Do not edit.\n")
    out.append(f"#pragma once\n#include \"mech_tables.h\"\n\n")
    sp = ", ".join(f'"{s}"' for s in M["species"])
    out.append(f"static const char* const {P}species[] = {{{sp}}};\n")
    out.append(_carr("double", P + "mw", M["mw"]))
    out.append(_carr("double", P + "imw", M["imw"]))
    out.append(_carr("double", P + "tmid", [t if t is not None else -1.0 for t in M["tmid"]]))
    for key, w in (("cv", 5), ("cp", 5), ("dcp", 4), ("u", 6), ("h", 6), ("g", 7)):
        vals = []
        for s in range(len(M["lo"])):
            vals += M["lo"][s][key] + M["hi"][s][key]
        out.append(_carr("double", P + "th_" + key, vals, w))
    rx = M["rxns"]

    def ints(f):
        return [f(r) for r in rx]

    def dbl(f):
        return [f(r) for r in rx]

    out.append(_carr("int", P + "rx_orig", ints(lambda r: r["orig"]), 16))
    out.append(_carr("int", P + "rx_kind", ints(lambda r: r["kind"]), 16))
    out.append(_carr("int", P + "rx_rev", ints(lambda r: r["rev"]), 16))
    out.append(_carr("double", P + "rx_A", dbl(lambda r: r["A"])))
    out.append(_carr("double", P + "rx_beta", dbl(lambda r: r["beta"])))
    out.append(_carr("double", P + "rx_EaR", dbl(lambda r: r["EaR"])))
    out.append(_carr("int", P + "rx_kcpow", ints(lambda r: r["kcpow"]), 16))
    out.append(_carr("double", P + "rx_sum_nuk", dbl(lambda r: r["sum_nuk"])))

    def padded(key, width, fill_sp=-1):
        sps, cs, ns = [], [], []
        for r in rx:
            lst = r[key]
            ns.append(len(lst))
            for j in range(width):
                if j < len(lst):
                    sps.append(lst[j][0])
                    cs.append(lst[j][1])
                else:
                    sps.append(fill_sp)
                    cs.append(0.0)
        return ns, sps, cs

    for key, width in (("fps", MAXPS), ("rps", MAXPS), ("kc", MAXKC), ("wup", MAXW), ("jn", MAXJN), ("hr", MAXPS), ("hp", MAXPS)):
        ns, sps, cs = padded(key, width)
        out.append(_carr("int", P + f"rx_{key}_n", ns, 16))
        out.append(_carr("int", P + f"rx_{key}_sp", sps, width))
        out.append(_carr("double", P + f"rx_{key}_c", cs, width))
    # efficiencies (CSR)
    off = [0]
    esp, ee, em1 = [], [], []
    for r in rx:
        for s, e, m1 in r["eff"]:
            esp.append(s)
            ee.append(e)
            em1.append(m1)
        off.append(len(esp))
    out.append(_carr("int", P + "eff_off", off, 16))
    out.append(_carr("int", P + "eff_sp", esp, 16))
    out.append(_carr("double", P + "eff_e", ee))
    out.append(_carr("double", P + "eff_m1", em1))
    # fall-off block: per reaction 16 doubles (zeros when not fall-off)
    # [P0, k0, beta0, EaR0, prdim, a, T3, T1, T2, oma, iT3, iT1, sriA, sriB, sriC, sriD]
    # and 8 ints [ntroe, p1, p2, j1, j2, j3, sri_n, sriE-present]
    fd, fi = [], []
    for r in rx:
        d = [0.0] * 17
        i = [0] * 8
        if "P0" in r:
            d[0:5] = [r["P0"], r["k0"], r["beta0"], r["EaR0"], r["prdim"]]
            if "troe" in r:
                t = r["troe"]
                d[5:12] = [t["a"], t["T3"], t["T1"], t["T2"], t["oma"], t["iT3"], t["iT1"]]
                i[0:6] = [t["n"], t["p1"], t["p2"], t["j1"], t["j2"], t["j3"]]
            if "sri" in r:
                d[12:17] = r["sri"]
                i[6] = r["sri_n"]
        fd += d
        fi += i
    out.append(_carr("double", P + "fo_d", fd, 17))
    out.append(_carr("int", P + "fo_i", fi, 8))
    if M["qss"]:
        qi = M["qss_info"]
        qs = ", ".join(f'"{q}"' for q in M["qss"])
        out.append(f"static const char* const {P}qss_species[] = {{{qs}}};\n")
        out.append(_carr("int", P + "q_rx", qi["q_rx"], 16))
        out.append(_carr("int", P + "q_off", qi["q_off"], 16))
        out.append(_carr("int", P + "q_term", qi["q_term"], 16))
        out.append(_carr("int", P + "q_role", qi["q_role"], 16))
        out.append(_carr("double", P + "q_coef", qi["q_coef"]))
        out.append(_carr("int", P + "rx_rmfwd", [r["rmf"] for r in M["rxns"]], 16))
    out.append(f"\nstatic const PPBMechTables ppbm_{cid} = {{\n")
    out.append(f'  "{name}", {nsp}, {nr},\n')
    fields = [
        "species", "mw", "imw", "tmid", "th_cv", "th_cp", "th_dcp", "th_u", "th_h", "th_g",
        "rx_orig", "rx_kind", "rx_rev", "rx_A", "rx_beta", "rx_EaR", "rx_kcpow", "rx_sum_nuk",
    ]
    for key in ("fps", "rps", "kc", "wup", "jn", "hr", "hp"):
        fields += [f"rx_{key}_n", f"rx_{key}_sp", f"rx_{key}_c"]
    fields += ["eff_off", "eff_sp", "eff_e", "eff_m1", "fo_d", "fo_i"]
    out.append("".join(f"  {P}{f},\n" for f in fields))
    if M["qss"]:
        qi = M["qss_info"]
        out.append(f"  {len(M['qss'])}, {len(qi['q_rx'])},\n")
        out.append("".join(f"  {P}{f},\n" for f in ("qss_species", "q_rx", "q_off", "q_term", "q_role", "q_coef",
                                                      "rx_rmfwd")))
    out.append("};\n")
    with open(path, "w") as fh:
        fh.write("".join(out))


def main(argv):
    ref = argv[1] if len(argv) > 1 else os.environ.get("PPB_REFERENCE_ROOT")
    if not ref:
        sys.exit(f"usage: python {argv[0]} REFERENCE_ROOT  (or set PPB_REFERENCE_ROOT): the PelePhysics tree")
    here = os.path.dirname(os.path.abspath(__file__))
    outdir = os.path.join(os.path.dirname(here), "csrc", "mech")
    os.makedirs(outdir, exist_ok=True)
    for m in MECHS:
        M = build(os.path.join(ref, "Mechanisms", m), m)
        emit_header(M, os.path.join(outdir, f"mech_{m}.h"))
        kinds = Counter(r["kind"] for r in M["rxns"])
        print(f"{m}: {len(M['species'])} species, {len(M['rxns'])} reactions, kinds {dict(kinds)}")


if __name__ == "__main__":
    main(sys.argv)
