"""SBML import: a mass-action SBML model -> the simulator's input folder.

The reference ships a Python 2 converter built on libsbml (SBML2BSW.py) that
writes `M_0` and `c_vector`, while the simulator reads `MX_0` and
`c_matrix` (one row per simulation); its feeds are always zero.  This
module needs no libsbml (the XML is read with the standard library) and
writes the files the simulator reads, with the same reaction semantics as
SBML2BSW.py (get_reactions):

* species in document order, named `name` (or `id`) + "_in_" + compartment
  (the `alphabet` file); initial amount = `initialAmount`, else
  `initialConcentration` (SBML2BSW.py get_initial_amounts);
* a reaction's rate constant(s): its kinetic law's local parameters, else
  the model parameters its formula names; two of them, or
  `reversible="true"`, add the reverse reaction right after it, with the
  second constant (SBML2BSW.py get_reactions);
* stoichiometries from the species references (default 1).

Differences, each a switch: species with `boundaryCondition="true"` or
`constant="true"` are written as feeds (`M_feed` = 1; the reference writes
zeros and leaves feeds as a TODO, `reference_feeds=True` restores that);
assignment rules and non-mass-action kinetics are rejected with an error
instead of being guessed.

    python -m cutauleaping_b200.sbml model.xml out_folder [--sims N]
        [--t-end T --samples K] [--reference-feeds]
"""
from __future__ import annotations

import argparse
import math
import os
import sys
import xml.etree.ElementTree as ET
from dataclasses import dataclass

import numpy as np


class SbmlError(ValueError):
    pass


@dataclass
class SbmlModel:
    names: list          # species labels (alphabet)
    x0: np.ndarray       # [S] initial amounts (float)
    feed: np.ndarray     # [S] 1 = held constant
    left: np.ndarray     # [R][S] reactant stoichiometry
    right: np.ndarray    # [R][S] product stoichiometry
    c: np.ndarray        # [R] rate constants
    reactions: list      # reaction labels


def _local(tag: str) -> str:
    return tag.rsplit("}", 1)[-1]


def _children(el, name):
    return [c for c in el if _local(c.tag) == name]


def _child(el, name):
    for c in el:
        if _local(c.tag) == name:
            return c
    return None


def _items(parent, listname, item):
    """Elements `item` of the list element `listname` under parent (none if absent)."""
    lst = _child(parent, listname)
    return [] if lst is None else _children(lst, item)


def _float(v, what):
    try:
        return float(v)
    except (TypeError, ValueError):
        raise SbmlError(f"{what}: not a number: {v!r}")


def _math_names(kl) -> list:
    """Identifiers (<ci>) of a kinetic law's MathML, in order of appearance."""
    math_el = _child(kl, "math")
    if math_el is None:
        return []
    return [(e.text or "").strip() for e in math_el.iter() if _local(e.tag) == "ci"]


def load(path: str, *, reference_feeds: bool = False) -> SbmlModel:
    try:
        root = ET.parse(path).getroot()
    except (ET.ParseError, OSError, LookupError, UnicodeError, ValueError) as e:
        raise SbmlError(f"cannot read SBML file {path}: {e}")
    model = _child(root, "model")
    if model is None:
        raise SbmlError(f"{path}: no <model> element")
    lst = _child(model, "listOfRules")
    if lst is not None and len(lst):
        raise SbmlError("rules (assignment / rate rules) are not supported")
    species = []
    for sp in _items(model, "listOfSpecies", "species"):
        sid = sp.get("id")
        label = sp.get("name") or sid
        if sp.get("compartment"):
            label = f"{label}_in_{sp.get('compartment')}"
        amount = sp.get("initialAmount")
        if amount is None or math.isnan(_float(amount, sid)):
            amount = sp.get("initialConcentration", "0")
        held = sp.get("boundaryCondition") == "true" or sp.get("constant") == "true"
        x0 = _float(amount, f"initial amount of {sid}")
        if not math.isfinite(x0):
            raise SbmlError(f"initial amount of {sid} is not finite")
        species.append((sid, label, x0, held))
    if not species:
        raise SbmlError("the model has no species")
    index = {sid: i for i, (sid, _, _, _) in enumerate(species)}
    params = {p.get("id"): _float(p.get("value"), f"parameter {p.get('id')}")
              for p in _items(model, "listOfParameters", "parameter") if p.get("value") is not None}
    S = len(species)
    left, right, c, labels = [], [], [], []
    for rx in _items(model, "listOfReactions", "reaction"):
        rid = rx.get("id") or rx.get("name") or f"R{len(labels)}"

        def side(listname):
            v = np.zeros(S, np.int64)
            for ref in _items(rx, listname, "speciesReference"):
                sp = ref.get("species")
                if sp not in index:
                    raise SbmlError(f"reaction {rid}: unknown species {sp}")
                st = _float(ref.get("stoichiometry", "1"), f"stoichiometry in {rid}")
                if not (0 <= st <= 127) or st != int(st):
                    raise SbmlError(f"reaction {rid}: stoichiometry must be an integer in [0, 127]")
                v[index[sp]] += int(st)
            return v
        lv, rv = side("listOfReactants"), side("listOfProducts")
        kl = _child(rx, "kineticLaw")
        if kl is None:
            raise SbmlError(f"reaction {rid}: no kinetic law")
        local = _items(kl, "listOfParameters", "parameter") + _items(kl, "listOfLocalParameters", "localParameter")
        local_vals = [_float(p.get("value"), f"local parameter of {rid}") for p in local]
        if local_vals:
            consts = local_vals
        else:
            named = []
            for n in _math_names(kl):
                if n in params and n not in named:
                    named.append(n)
            if not named:
                raise SbmlError(f"reaction {rid}: no kinetic parameter found")
            consts = [params[n] for n in named]
        if not all(math.isfinite(k) and k >= 0 for k in consts):
            raise SbmlError(f"reaction {rid}: rate constants must be finite and >= 0")
        reverse = rx.get("reversible") == "true" or len(consts) == 2
        if len(consts) > 2 or (reverse and len(consts) != 2) or len(consts) == 0:
            raise SbmlError(f"reaction {rid}: expected one rate constant (two if reversible), "
                            f"found {len(consts)}")
        left.append(lv), right.append(rv), c.append(consts[0]), labels.append(rid)
        if reverse:
            left.append(rv), right.append(lv), c.append(consts[1]), labels.append(rid + " (reverse)")
    if not left:
        raise SbmlError("the model has no reactions")
    feed = np.array([0 if reference_feeds else int(h) for (_, _, _, h) in species], np.int32)
    return SbmlModel([lab for (_, lab, _, _) in species], np.array([a for (_, _, a, _) in species]), feed,
                     np.array(left, np.int32), np.array(right, np.int32), np.array(c, np.float64), labels)


def _fmt(v: float) -> str:
    return repr(float(v)) if v != int(v) or abs(v) >= 1e16 else str(int(v))


def write_folder(m: SbmlModel, out: str, *, sims: int = 1, t_end: float | None = None,
                 samples: int | None = None) -> str:
    """Write the input folder: left_side, right_side, M_feed, MX_0 and
    c_matrix (`sims` identical rows), alphabet, and t_vector when t_end and
    samples are given (instants t_end*i/samples, i = 1..samples)."""
    os.makedirs(out, exist_ok=True)

    def rows(name, M):
        with open(os.path.join(out, name), "w") as f:
            for r in np.atleast_2d(M):
                f.write("\t".join(_fmt(v) for v in r) + "\n")
    x0 = np.rint(m.x0)
    if (x0 < 0).any() or (x0 > 2**31 - 1).any():
        raise SbmlError("initial amounts must be counts in [0, 2^31)")
    rows("left_side", m.left)
    rows("right_side", m.right)
    rows("M_feed", m.feed.reshape(1, -1))
    rows("MX_0", np.tile(x0, (sims, 1)))
    rows("c_matrix", np.tile(m.c, (sims, 1)))
    with open(os.path.join(out, "alphabet"), "w") as f:
        f.write("\t".join(m.names) + "\n")
    if t_end is not None and samples:
        with open(os.path.join(out, "t_vector"), "w") as f:
            f.write("".join(repr(float(t_end * i / samples)) + "\n" for i in range(1, samples + 1)))
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="SBML (mass-action) -> cuTauLeaping input folder")
    ap.add_argument("sbml")
    ap.add_argument("out")
    ap.add_argument("--sims", type=int, default=1, help="rows of MX_0 / c_matrix")
    ap.add_argument("--t-end", type=float, default=None)
    ap.add_argument("--samples", type=int, default=None)
    ap.add_argument("--reference-feeds", action="store_true", help="write M_feed zeros as SBML2BSW.py does")
    a = ap.parse_args(argv)
    try:
        m = load(a.sbml, reference_feeds=a.reference_feeds)
        write_folder(m, a.out, sims=a.sims, t_end=a.t_end, samples=a.samples)
    except SbmlError as e:
        print(f"ERROR: {e}", file=sys.stderr)
        return 2
    print(f" * {len(m.names)} species, {len(m.c)} reactions -> {a.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
