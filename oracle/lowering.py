"""Independent restatement of the model lowering for the configuration
subset the workloads use (test infrastructure: the checker of the
library's lowering, never imported by the product).

It reads config.yml with PyYAML and restates, without the library's C++
front end, what the reference builds from it:
  - the allowed (2S+1, L) waves of each two-body vertex by LS coupling with
    parity conservation and the identical-daughter rule (-1)^(L+S) = +1 for
    bosons (src/AmpGen.cu:69-129);
  - the amplitudes: decay chains in file order, per chain the intermediate
    groups (J, P) and their resonances in listed order, per resonance the
    product of its vertices' waves (top vertex outermost), named
    "Mother→a+b_SL(2S+1,L)_R→c+d_SL(2S+1,L)" with the chain's tags replaced
    by the resonance name (src/Info.cu:285-299);
  - the free resonance parameters: per resonance at its first appearance,
    the parameters listed in `free` (all for `[-1]` and for custom
    lineshapes), named "<resonance>_<parameter>" (src/Info.cu:86-98), with
    `free_range` bounds or the default +-50 % of the value;
  - one free complex coupling per amplitude (no coupling matrix);
  - `Constraints: var_equal` groups of resonance parameters: the later
    members share the first one's slot and are not free parameters of their
    own;
  - the parent's `polarization` list of m values: the polarisation states
    kept, as indices into m = +J .. -J (src/Analysis.cu:4249-4322).
Supported lineshapes: BWR (mass, width) and Custom (paramNames). Anything
else raises NotImplementedError, so a test cannot pass by omission.
"""
from fractions import Fraction

import yaml


class _Loader(yaml.SafeLoader):
    """SafeLoader whose mappings accept sequence keys (the intermediates'
    `[J: 1, P: -1]` group keys) as tuples of (key, value) pairs."""


def _construct_mapping(loader, node, deep=False):
    out = {}
    for key_node, value_node in node.value:
        key = loader.construct_object(key_node, deep=True)
        if isinstance(key, list):
            items = []
            for k in key:
                items.extend(k.items() if isinstance(k, dict) else [(k, None)])
            key = tuple(items)
        out[key] = loader.construct_object(value_node, deep=True)
    return out


_Loader.add_constructor(yaml.resolver.BaseResolver.DEFAULT_MAPPING_TAG, _construct_mapping)


def _twice(j):
    """2J as an integer (J integer or half-integer)."""
    t = Fraction(str(j)) * 2
    if t.denominator != 1:
        raise ValueError(f"spin {j} is not a multiple of 1/2")
    return int(t)


def ls_waves(j0, p0, j1, p1, j2, p2, identical=False):
    """Allowed (2S+1, L) of the decay j0 -> j1 + j2 (spins J, parities +-1):
    S from |J1 - J2| to J1 + J2, L from |J0 - S| to J0 + S, kept when
    P0 = P1 P2 (-1)^L and, for identical daughters, (-1)^(L+S) = +1 (bosons,
    integer spin) or -1 (fermions). Ordered by S, then L."""
    a, b, c = _twice(j0), _twice(j1), _twice(j2)
    boson = b % 2 == 0
    waves = []
    for two_s in range(abs(b - c), b + c + 1, 2):
        for two_l in range(abs(a - two_s), a + two_s + 1, 2):
            if two_l % 2:
                continue  # half-integer L cannot occur for a consistent spin set
            ell, s = two_l // 2, two_s // 2
            if p0 != p1 * p2 * (-1) ** ell:
                continue
            if identical and ((ell + s) % 2 == 0) != boson:
                continue
            waves.append((two_s + 1, ell))
    return waves


def _param_names(res):
    model = str(res.get("model", "")).lower()
    if model == "bwr":
        return ["mass", "width"], list(res["parameters"])
    if model == "custom":
        return list(res["paramNames"]), list(res["paramValues"])
    raise NotImplementedError(f"lineshape {res.get('model')!r} is outside the restated subset")


def lower(config_path):
    """{"amplitude_names", "slots" [(name, init, lower, upper)], "n_free"} of a config."""
    with open(config_path) as f:
        cfg = yaml.load(f, Loader=_Loader)
    particles = cfg["Particles"]
    resonances = cfg["Resonances"]
    identical = set()
    for pair in (cfg.get("Constraints") or {}).get("identical", []) or []:
        identical.add(frozenset(pair))
    for key in ("CouplingMatrix", "coupling_matrix"):
        if key in cfg:
            raise NotImplementedError(f"{key} is outside the restated subset")
    tied = set()
    for group in (cfg.get("Constraints") or {}).get("var_equal", []) or []:
        tied.update(group[1:])

    names, slots, seen = [], [], set()
    for chain_name, chain in cfg["DecayChains"].items():
        inter = chain["intermediates"]
        steps = [(m, d) for m, d in chain.items() if m != "intermediates"]
        # the top vertex: a mother that is a particle, decaying to [[bachelor, tag]]
        top = [(m, d) for m, d in steps if m in particles]
        if len(top) != 1 or len(inter) != 1:
            raise NotImplementedError(f"chain {chain_name}: one top vertex and one intermediate expected")
        mother, (tdaus,) = top[0][0], top[0][1]
        tag = next(iter(inter))
        bdaus = chain[tag]
        jm, pm = particles[mother]["J"], particles[mother]["P"]
        for group in inter[tag]:
            ((jp, reslist),) = group.items()
            jp = dict(jp)
            jr, pr = jp["J"], jp["P"]
            for rname in reslist:
                def spin_parity(x):
                    return (jr, pr) if x == tag else (particles[x]["J"], particles[x]["P"])
                (j1, p1), (j2, p2) = spin_parity(tdaus[0]), spin_parity(tdaus[1])
                top_waves = ls_waves(jm, pm, j1, p1, j2, p2, identical=frozenset(tdaus) in identical)
                (k1, q1), (k2, q2) = spin_parity(bdaus[0]), spin_parity(bdaus[1])
                bot_waves = ls_waves(jr, pr, k1, q1, k2, q2, identical=frozenset(bdaus) in identical)
                rep = lambda x: rname if x == tag else x  # noqa: E731
                for st, lt in top_waves:
                    for sb, lb in bot_waves:
                        names.append(f"{mother}→{rep(tdaus[0])}+{rep(tdaus[1])}_SL({st},{lt})_"
                                     f"{rname}→{bdaus[0]}+{bdaus[1]}_SL({sb},{lb})")
                if rname in seen:
                    continue
                seen.add(rname)
                res = resonances[rname]
                pnames, pvals = _param_names(res)
                free = res.get("free")
                custom = str(res.get("model", "")).lower() == "custom"
                if free is None:
                    idx = list(range(len(pnames))) if custom else []
                elif list(free) == [-1]:
                    idx = list(range(len(pnames)))
                else:
                    idx = [i for i in range(len(pnames)) if i in set(free)]
                ranges = res.get("free_range")
                for n_i, i in enumerate(idx):
                    v = float(pvals[i])
                    if ranges:
                        lo, hi = (float(x) for x in ranges[n_i])
                    else:
                        lo, hi = v - 0.5 * abs(v), v + 0.5 * abs(v)
                    if f"{rname}_{pnames[i]}" not in tied:
                        slots.append((f"{rname}_{pnames[i]}", v, lo, hi))
    # polarisation states: the parent's m = +J .. -J times the spin states of
    # the (massive) final-state particles; a parent's `polarization` list
    # keeps some of its m values
    parent = particles[mother]
    two_j = _twice(parent["J"])
    n_final = 1
    for name in cfg["Data"]["order"]:
        fp = particles[name]
        if _twice(fp["J"]) and not float(fp.get("mass", 0.0)) > 0.0:
            raise NotImplementedError("massless final-state particles with spin are outside the restated subset")
        n_final *= _twice(fp["J"]) + 1
    pols = parent.get("polarization")
    if pols is None:
        pol_map = list(range((two_j + 1) * n_final))
    elif n_final == 1:
        pol_map = [int((two_j - _twice(m)) // 2) for m in pols]
    else:
        raise NotImplementedError("a polarisation list with spinning final-state particles is outside the subset")
    return {"amplitude_names": names, "slots": slots, "n_free": len(names), "npol": len(pol_map),
            "npol_total": (two_j + 1) * n_final, "pol_map": pol_map}
