"""CHEMKIN mechanism, thermodynamic and transport data -> the species and
reaction tables of the path (cfd::Species / cfd::Reaction, src/ChemData.h).

A restatement of src/ChemData.cpp:11-685 and src/Element.cpp, keeping its
behaviours because they change the tables the kernels see:

* species are numbered in order of appearance in the SPECIES block (A15);
* the THERMO header range line does not override the defaults 300/1000/5000 K
  (ChemData.cpp:147-151 resizes vectors that already have that size); only
  the per-species columns 45-75 set T_low / T_high / T_mid;
* molecular weights sum element weights in element-name order (std::map);
* Arrhenius Ea is divided by R_c, but LOW and REV Ea are used as given (A7);
* DUPLICATE pairs merge into one reaction of type 3 whose second Arrhenius
  set is the partner's (ChemData.cpp:457-495, A14); TROE with 3 numbers is
  type 6, with 4 numbers type 7; "+M" gives type 4, "(+M)" type 5.

The tables are returned as numpy arrays keyed like the fields of ostc_param.
"""
from __future__ import annotations

import json
import math
import re
from pathlib import Path
from typing import Dict, List

import numpy as np

try:
    from ostc import Mechanism
except ImportError:  # pragma: no cover
    Mechanism = None

R_C = 1.98720425864083  # cal/(mol K), src/Constants.h:19
BOLTZMANN = 1.380649e-23

# atomic weights of src/Element.cpp (the elements a CHEMKIN H/C/N/O/Ar mechanism uses)
ATOMIC_WEIGHT = {"H": 1.008, "HE": 4.002602, "C": 12.011, "N": 14.007, "O": 15.999, "AR": 39.95, "F": 18.998403163,
                 "NE": 20.1797, "S": 32.06, "CL": 35.45, "D": 2.0141017781, "TR": 3.0160492820}


def _tokens_after(text: str, keys) -> List[str]:
    return text


def read_species(mech_text: str):
    """ELEMENTS and SPECIES blocks (ChemData.cpp:11-76)."""
    toks = []
    for line in mech_text.splitlines():
        toks_line = line.split()
        for t in toks_line:
            if t.startswith("!"):
                break
            toks.append(t)
    it = iter(toks)
    for t in it:
        if t in ("ELEMENTS", "ELEM"):
            break
    elems: List[str] = []
    for t in it:
        u = t.upper()
        if u == "END":
            continue
        if u in ("SPECIES", "SPEC"):
            break
        elems.append(u)
    species: List[str] = []
    for t in it:
        u = t.upper()
        if u == "END":
            continue
        if u in ("REACTIONS", "REAC", "THERMO"):
            break
        if u not in species:
            species.append(u)
    return elems, species


def read_therm(therm_text: str, species: List[str], elems: List[str]):
    """THERMO records (ChemData.cpp:131-290)."""
    ns = len(species)
    idx = {s: i for i, s in enumerate(species)}
    t_low = np.full(ns, 300.0)
    t_mid = np.full(ns, 1000.0)
    t_high = np.full(ns, 5000.0)
    hi = np.zeros((ns, 7))
    lo = np.zeros((ns, 7))
    mw = np.zeros(ns)
    lines = therm_text.splitlines()
    p = 0
    while p < len(lines) and "THERMO" not in lines[p].upper():
        p += 1
    p += 1
    while p < len(lines) and (not lines[p].strip() or lines[p].startswith("!")):
        p += 1
    p += 1  # the global temperature-range line (no effect, see module docstring)
    have = set()
    while p < len(lines):
        line = lines[p]
        if not line.strip() or line.startswith("!"):
            p += 1
            continue
        key = line.upper().split()[0]
        if key == "END":
            p += 1
            continue
        if key in ("REACTIONS", "TRANSPORT", "TRAN") or len(have) >= ns:
            break
        name = line[:18].upper().split()[0] if line[:18].split() else ""
        if name not in idx or idx[name] in have:
            p += 4
            continue
        k = idx[name]
        t_low[k] = float(line[45:55])
        t_high[k] = float(line[55:65])
        tm = line[65:75].split()
        if tm:
            t_mid[k] = float(tm[0])
        comp = {}
        for i in range(4):
            field = line[24 + 5 * i:29 + 5 * i].lstrip()
            if not field or field.startswith("0"):
                break
            parts = field.split()
            el = parts[0].upper()
            if el not in elems:
                continue
            comp[el] = int(parts[1]) if len(parts) > 1 else 0
        w = 0.0
        for el in sorted(elems):  # std::map<std::string,int> iteration order
            w += ATOMIC_WEIGHT[el] * comp.get(el, 0)
        mw[k] = w
        l1, l2, l3 = lines[p + 1], lines[p + 2], lines[p + 3]
        c = [float(l1[15 * q:15 * q + 15]) for q in range(5)]
        d = [float(l2[15 * q:15 * q + 15]) for q in range(5)]
        e = [float(l3[15 * q:15 * q + 15]) for q in range(4)]
        hi[k, :5] = c
        hi[k, 5:7] = d[:2]
        lo[k, :3] = d[2:5]
        lo[k, 3:7] = e
        have.add(k)
        p += 4
    return dict(t_low=t_low, t_mid=t_mid, t_high=t_high, high_temp_coeff=hi, low_temp_coeff=lo, mw=mw)


def _reduced_dipole(i, mu, eps, sigma):  # ChemData.cpp:405-416
    if mu[i] == 0:
        return 0.0
    debye = 1e-18 * math.sqrt(1e-7)
    cm_a = math.pow(1e8, 1.5)
    conv = debye * cm_a / math.sqrt(BOLTZMANN)
    return conv * mu[i] / math.sqrt(eps[i] * sigma[i] * sigma[i] * sigma[i])


def read_tran(tran_text: str, species: List[str], mw: np.ndarray):
    """TRANSPORT records and the derived mixing constants (ChemData.cpp:292-402)."""
    ns = len(species)
    idx = {s: i for i, s in enumerate(species)}
    eps = np.zeros(ns)
    sig = np.zeros(ns)
    mu = np.zeros(ns)
    alp = np.zeros(ns)
    LJ = np.zeros(ns)
    vc = np.zeros(ns)
    have = set()
    for line in tran_text.splitlines():
        if not line.strip() or line.startswith("!"):
            continue
        t = line.upper().split()
        if t[0].startswith(("END", "REACTIONS", "REAC")):
            break
        if t[0] not in idx:
            continue
        if len(have) >= ns:
            break
        k = idx[t[0]]
        if k in have:
            continue
        eps[k], sig[k], mu[k], alp[k] = float(t[2]), float(t[3]), float(t[4]), float(t[5])
        LJ[k] = 1.0 / eps[k]
        vc[k] = 2.6693e-6 * math.sqrt(mw[k]) / (sig[k] * sig[k])
        have.add(k)
    W4 = np.zeros((ns, ns))
    S8 = np.zeros((ns, ns))
    for i in range(ns):
        for j in range(ns):
            W4[i, j] = math.pow(mw[j] / mw[i], 0.25)
            S8[i, j] = 1.0 / math.sqrt(8 * (1 + mw[i] / mw[j]))
    bdc = np.zeros((ns, ns))
    kbe = np.zeros((ns, ns))
    for j in range(ns):
        for k in range(j + 1, ns):
            Wjk = mw[j] * mw[k] / (mw[j] + mw[k])
            xi = 1.0
            if (mu[j] != 0) != (mu[k] != 0):  # compute_xi, ChemData.cpp:386-403
                p_, n_ = (j, k) if mu[j] != 0 else (k, j)
                a_n = alp[n_] / math.pow(sig[n_], 3)
                mp = _reduced_dipole(p_, mu, eps, sig)
                xi = 1.0 + 0.25 * a_n * mp * mp * math.sqrt(eps[p_] / eps[n_])
            s_jk = 0.5 * (sig[j] + sig[k]) * math.pow(xi, -1.0 / 6.0)
            bdc[j, k] = bdc[k, j] = 0.0188324 / (math.sqrt(Wjk) * s_jk * s_jk)
            e_jk = xi * xi * math.sqrt(eps[j] * eps[k])
            kbe[j, k] = kbe[k, j] = 1.0 / e_jk
    return dict(LJ_potent_inv=LJ, vis_coeff=vc, WjDivWi_to_One4th=W4, sqrt_WiDivWjPl1Mul8=S8,
                binary_diffusivity_coeff=bdc, kb_over_eps_jk=kbe)


def _parse_side(s: str, idx: Dict[str, int], ns: int):
    """'2H+O2' -> stoichiometry vector, following read_reaction_line's split
    (a leading digit is the coefficient; '++' keeps a '+' in a name)."""
    nu = np.zeros(ns, dtype=np.int32)
    order = 0
    rest = s
    while True:
        p = rest.find("+")
        if p < 0:
            break
        if p + 1 < len(rest) and rest[p + 1] == "+":
            p += 1
        c = 1
        if rest[0].isdigit():
            c = int(rest[0])
            rest = rest[1:]
            name = rest[:p - 1]
        else:
            name = rest[:p]
        nu[idx[name]] += c
        order += c
        rest = rest[len(name) + 1:]
    c = 1
    if rest and rest[0].isdigit():
        c = int(rest[0])
        rest = rest[1:]
    nu[idx[rest]] += c
    order += c
    return nu, order


def read_reactions(mech_text: str, species: List[str]):
    """REACTIONS block (ChemData.cpp:418-685)."""
    ns = len(species)
    idx = {s: i for i, s in enumerate(species)}
    lines = mech_text.splitlines()
    p = 0
    while p < len(lines) and not re.match(r"^\s*(REACTIONS|REAC)\b", lines[p]):
        p += 1
    p += 1
    R: List[dict] = []
    dup_open: List[int] = []

    def new():
        return dict(label=1, nuf=np.zeros(ns, np.int32), nub=np.zeros(ns, np.int32), order=0, A=0.0, b=0.0, Ea=0.0,
                    A2=0.0, b2=0.0, Ea2=0.0, tb=np.ones(ns), ta=0.0, t3=0.0, t1=0.0, t2=0.0)

    line = lines[p].upper() if p < len(lines) else "END"
    while line.strip() != "END":
        if not line.strip() or line.startswith("!"):
            p += 1
            line = lines[p].upper() if p < len(lines) else "END"
            continue
        r = new()
        text = line
        if "+M" in text:
            r["label"] = 4
            lp = text.find("(+")
            if lp >= 0:
                r["label"] = 5
                rp = text.find(")", lp)
                text = text[:lp] + text[rp + 1:]
                lp = text.find("(+")
                rp = text.rfind(")")
                text = text[:lp] + text[rp + 1:]
            else:
                q = text.find("+M")
                text = text[:q] + text[q + 2:]
                q = text.find("+M")
                text = text[:q] + text[q + 2:]
        it_s = text.find("<")
        if it_s < 0:
            it_s = text.find("=")
        text = text[:it_s + 1].replace(" ", "<") + text[it_s + 1:]
        toks = text.split()
        eq, r["A"], r["b"], r["Ea"] = toks[0], float(toks[1]), float(toks[2]), float(toks[3]) / R_C
        it_s, it_e, it_b = eq.find("<"), eq.find("="), eq.find(">")
        if it_s < 0:
            if it_b >= 0:
                r["label"] = 0
            else:
                it_b = it_e
            it_s = it_e
        nuf, of = _parse_side(eq[:it_s], idx, ns)
        nub, ob = _parse_side(eq[it_b + 1:], idx, ns)
        r["nuf"], r["nub"], r["order"] = nuf, nub, ob - of
        # auxiliary lines (get_auxi_info, ChemData.cpp:630-685)
        is_dup = False
        p += 1
        while p < len(lines):
            raw = lines[p].upper()
            aux = raw.replace("/", " ")
            t = aux.split()
            if raw.startswith("!") or not raw.strip():
                p += 1
                continue
            if t[0] == "END" or "=" in raw:
                break
            p += 1
            if t[0] == "PLOG":
                continue
            if t[0] in ("DUPLICATE", "DUP"):
                is_dup = True
                r["label"] = 3
                continue
            if t[0] == "REV":
                r["A2"], r["b2"], r["Ea2"] = float(t[1]), float(t[2]), float(t[3])
                r["label"] = 2
            elif t[0] == "LOW":
                r["A2"], r["b2"], r["Ea2"] = float(t[1]), float(t[2]), float(t[3])
            elif t[0] == "TROE":
                r["label"] = 6
                r["ta"], r["t3"], r["t1"] = float(t[1]), float(t[2]), float(t[3])
                if len(t) > 4:
                    r["t2"] = float(t[4])
                    r["label"] = 7
            else:
                for q in range(0, len(t) - 1, 2):
                    r["tb"][idx[t[q]]] = float(t[q + 1])
        line = lines[p].upper() if p < len(lines) else "END"
        if is_dup:
            partner = None
            for q, d in enumerate(dup_open):
                if np.array_equal(R[d]["nuf"], r["nuf"]) and np.array_equal(R[d]["nub"], r["nub"]):
                    partner = q
                    break
            if partner is not None:
                d = dup_open.pop(partner)
                R[d]["A2"], R[d]["b2"], R[d]["Ea2"] = r["A"], r["b"], r["Ea"]
                continue
            dup_open.append(len(R))
        R.append(r)
    nr = len(R)
    out = dict(
        reac_type=np.array([r["label"] for r in R], np.int32),
        stoi_f=np.array([r["nuf"] for r in R], np.int32).reshape(nr, ns),
        stoi_b=np.array([r["nub"] for r in R], np.int32).reshape(nr, ns),
        reac_order=np.array([r["order"] for r in R], np.int32),
        third_body_coeff=np.array([r["tb"] for r in R]).reshape(nr, ns),
    )
    for key, src in (("A", "A"), ("b", "b"), ("Ea", "Ea"), ("A2", "A2"), ("b2", "b2"), ("Ea2", "Ea2"),
                     ("troe_alpha", "ta"), ("troe_t3", "t3"), ("troe_t1", "t1"), ("troe_t2", "t2")):
        out[key] = np.array([r[src] for r in R], np.float64)
    return out


def load_chemkin(mech: Path, therm: Path, tran: Path, reactions: bool = True):
    mech_text = Path(mech).read_text()
    elems, species = read_species(mech_text)
    tab = read_therm(Path(therm).read_text(), species, elems)
    tab.update(read_tran(Path(tran).read_text(), species, tab["mw"]))
    nr = 0
    if reactions:
        rt = read_reactions(mech_text, species)
        tab.update(rt)
        nr = len(rt["reac_type"])
    return Mechanism(species, tab, nr)


def save_json(mech, path: Path):
    data = {"species": mech.names, "n_reac": mech.n_reac,
            "tables": {k: {"dtype": str(v.dtype), "shape": list(v.shape), "data": v.ravel().tolist()}
                       for k, v in mech.tables.items()}}
    Path(path).write_text(json.dumps(data, indent=0))


def load_json(path: Path):
    data = json.loads(Path(path).read_text())
    tab = {k: np.array(v["data"], dtype=v["dtype"]).reshape(v["shape"]) for k, v in data["tables"].items()}
    return Mechanism(data["species"], tab, data["n_reac"])


DATA = Path(__file__).resolve().parent / "data"


def h2_air_9sp():
    """The 9-species, 19-reaction H2-air mechanism of the reacting workload
    (tables generated by data/make_mechanism.py from the CHEMKIN inputs)."""
    return load_json(DATA / "h2_air_9sp.json")


def h2_mixing_4sp():
    """The reference's non-reacting 4-species set (H2, H2O, O2, N2 in the
    order of input_files/chemistry/H2_mech_mixing.inp, with therm.dat and
    tran.dat; the reference reads no reactions for it, reaction = 0)."""
    return load_json(DATA / "h2_mixing_4sp.json")


_SPECIES_TABS = ("t_low", "t_mid", "t_high", "high_temp_coeff", "low_temp_coeff", "mw", "LJ_potent_inv", "vis_coeff")
_PAIR_TABS = ("WjDivWi_to_One4th", "sqrt_WiDivWjPl1Mul8", "binary_diffusivity_coeff", "kb_over_eps_jk")
_REAC_SPECIES_TABS = ("stoi_f", "stoi_b", "third_body_coeff")


def with_inert_copies(mech, name: str, k: int):
    """The mechanism with k more species that are inert copies of `name`
    (same thermodynamic and transport data, pair data of the copied pairs,
    never reacting, third-body efficiency of the original), appended after
    the others as name_1 .. name_k: mechanisms of any species count up to
    OSTC_MAX_SPEC for the tests of the per-count builds."""
    import numpy as np

    src = mech.names.index(name)
    ix = list(range(mech.n_spec)) + [src] * k
    tab = {}
    for key, v in mech.tables.items():
        if key in _SPECIES_TABS:
            tab[key] = np.ascontiguousarray(v[ix])
        elif key in _PAIR_TABS:
            tab[key] = np.ascontiguousarray(v[np.ix_(ix, ix)])
        elif key in ("stoi_f", "stoi_b"):
            tab[key] = np.ascontiguousarray(np.concatenate([v, np.zeros((v.shape[0], k), v.dtype)], axis=1))
        elif key == "third_body_coeff":
            tab[key] = np.ascontiguousarray(v[:, ix])
        else:
            tab[key] = v.copy()
    return type(mech)(mech.names + ["%s_%d" % (name, q + 1) for q in range(k)], tab, mech.n_reac)


def subset(mech, keep: List[str], reactions: bool = True):
    """The mechanism restricted to the species `keep` (in that order) and,
    with reactions, to the reactions whose reactants and products are all
    kept (third-body efficiencies of dropped species are dropped with them).
    Species and pair tables are the same numbers, re-indexed: what the
    reference's parser builds for a mechanism file listing those species."""
    import numpy as np

    ix = [mech.names.index(n) for n in keep]
    tab = {}
    for k in _SPECIES_TABS:
        tab[k] = np.ascontiguousarray(mech.tables[k][ix])
    for k in _PAIR_TABS:
        tab[k] = np.ascontiguousarray(mech.tables[k][np.ix_(ix, ix)])
    nr = 0
    if reactions and mech.n_reac:
        drop = [i for i in range(mech.n_spec) if i not in ix]
        sf, sb = mech.tables["stoi_f"], mech.tables["stoi_b"]
        rows = [r for r in range(mech.n_reac) if not any(sf[r, d] or sb[r, d] for d in drop)]
        for k, v in mech.tables.items():
            if k in _SPECIES_TABS or k in _PAIR_TABS:
                continue
            v = v[rows]
            if k in _REAC_SPECIES_TABS:
                v = v[:, ix]
            tab[k] = np.ascontiguousarray(v)
        nr = len(rows)
    return type(mech)(list(keep), tab, nr)
