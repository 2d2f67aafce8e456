"""Reaction-network text format: a writer for synthetic networks and a parser.

The file format is VULCAN's (reference `network.py:103-105`, `:262-301`):

    <id> [ A + 2*B + M -> C + D ]  <a> <n> <E> ...

with section markers (`# 3-body`, `# photo`, ...) and a `# reverse stops`
marker. The parser here is this package's own and produces the same padded
stoichiometry tables as the reference parser (`network.py:197-491`):

* reactions are 1-based; the forward reaction of the k-th record sits at
  row ``2k-1`` and its reverse at row ``2k`` with the two sides swapped
  (reference `network.py:403-419`);
* repeated species on one side are collapsed into one slot whose stoichiometry
  is the sum, slots ordered by first appearance on that side (`:270-284`);
* `M` is dropped from the slots and recorded per direction as a three-body flag
  (`:286-291`, `:424-425`);
* unused slots hold the padding index ``ni`` with stoichiometry 0 (`:377-385`);
* species are numbered by first appearance in the file (`:223-229`);
* the leading numeric columns give the rate parameters: ``a n E`` in the
  two-body and both three-body sections, plus ``a_inf n_inf E_inf`` in the
  three-body section with high-pressure rates (`:444-451`); every row of a
  section carries its flag (`:427-443`); ``stop_rev_indx`` is the row of the
  `# reverse stops` marker, else the first photo row, else ``nr + 1``
  (`:252-253`, `:353-356`).

Config-named extra species (reference `network.py:157-194`) are not appended:
the synthetic networks name every species in their reactions.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

import numpy as np

_LINE = re.compile(r"^\s*(\d+)\s*\[\s*([^\]]+)\s*\]\s*(.*)$")

TWO_BODY = "two_body"
THREE_BODY_KINF = "three_body_kinf"
THREE_BODY_NO_KINF = "three_body_no_kinf"
SPECIAL = "special"
CONDEN = "conden"
RADIATIVE = "radiative"
PHOTO = "photo"
ION = "ion"


@dataclass
class NetworkTables:
    """Padded stoichiometry tables of a parsed network (host, NumPy).

    Shapes follow the reference `Network` (`network.py:36-100`): every table
    has ``nr + 1`` rows, row 0 unused.
    """

    species: tuple
    ni: int
    nr: int
    reactant_idx: np.ndarray     # int64 [nr+1, T]
    product_idx: np.ndarray      # int64 [nr+1, T]
    reactant_stoich: np.ndarray  # float64 [nr+1, T]
    product_stoich: np.ndarray   # float64 [nr+1, T]
    is_three_body: np.ndarray    # bool [nr+1]
    is_photo: np.ndarray         # bool [nr+1]
    pho_rate_index: dict = field(default_factory=dict)  # (species, branch) -> row
    photo_sp: tuple = ()
    # rate parameters and section flags ([nr+1]; None for tables built by hand)
    a: np.ndarray = None
    n: np.ndarray = None
    E: np.ndarray = None
    a_inf: np.ndarray = None
    n_inf: np.ndarray = None
    E_inf: np.ndarray = None
    is_forward: np.ndarray = None
    has_kinf: np.ndarray = None
    is_special: np.ndarray = None
    is_conden: np.ndarray = None
    is_radiative: np.ndarray = None
    is_ion: np.ndarray = None
    stop_rev_indx: int = 0
    Rf: dict = field(default_factory=dict)              # forward row -> "A + B -> C + D"

    @property
    def max_terms(self) -> int:
        return int(self.reactant_idx.shape[1])


def _section_of(line: str):
    s = line.lstrip()
    if s.startswith("# 3-body reactions without high-pressure rates"):
        return THREE_BODY_NO_KINF
    if s.startswith("# 3-body"):
        return THREE_BODY_KINF
    if s.startswith("# special"):
        return SPECIAL
    if s.startswith("# condensation"):
        return CONDEN
    if s.startswith("# radiative"):
        return RADIATIVE
    if s.startswith("# photo"):
        return PHOTO
    if s.startswith("# ionisation") or s.startswith("# ionization"):
        return ION
    return None


def _side(text: str):
    out = []
    for term in text.split("+"):
        term = term.strip()
        if not term:
            continue
        if "*" in term:
            c, sp = term.split("*", 1)
            out.append((int(c), sp.strip()))
        else:
            out.append((1, term))
    return out


def parse_network_text(text: str) -> NetworkTables:
    """Parse network-file text into `NetworkTables`."""
    order: list[str] = []
    index: dict[str, int] = {}
    records = []
    section = TWO_BODY
    photo_sp: list[str] = []
    pho_rate_index: dict = {}

    def intern(sp: str) -> None:
        if sp != "M" and sp not in index:
            index[sp] = len(order)
            order.append(sp)

    row = 1
    stop_rev = None
    photo_row = None
    for raw in text.splitlines():
        if not raw.strip():
            continue
        sec = _section_of(raw)
        if sec is not None:
            section = sec
            if sec == PHOTO and photo_row is None:
                photo_row = row
            continue
        if raw.lstrip().startswith("# reverse stops"):
            stop_rev = row
            continue
        if raw.lstrip().startswith("#"):
            continue
        m = _LINE.match(raw)
        if m is None:
            continue
        eq, tail = m.group(2).strip(), m.group(3)
        if "->" not in eq:
            raise ValueError(f"reaction without '->': {eq!r}")
        lhs, rhs = eq.split("->", 1)
        reac, prod = _side(lhs), _side(rhs)
        for _, sp in reac + prod:
            intern(sp)

        def collapse(terms):
            acc: dict[int, float] = {}
            for c, sp in terms:
                if sp == "M":
                    continue
                acc[index[sp]] = acc.get(index[sp], 0.0) + float(c)
            return acc

        cols = tail.split()
        nums = []
        for c in cols:
            try:
                nums.append(float(c))
            except ValueError:
                break
        rec = dict(row=row, section=section, reac=collapse(reac), prod=collapse(prod),
                   m_reac=any(sp == "M" for _, sp in reac),
                   m_prod=any(sp == "M" for _, sp in prod), eq=eq, nums=nums)
        records.append(rec)
        if section == PHOTO:
            target = cols[0] if cols else eq.split()[0]
            if target not in photo_sp:
                photo_sp.append(target)
            if len(cols) >= 2 and cols[1].isdigit():
                pho_rate_index[(cols[0], int(cols[1]))] = row
        row += 2

    nr = row - 1
    ni = len(order)
    T = max([1] + [len(r["reac"]) for r in records] + [len(r["prod"]) for r in records])
    r_idx = np.full((nr + 1, T), ni, dtype=np.int64)
    p_idx = np.full((nr + 1, T), ni, dtype=np.int64)
    r_st = np.zeros((nr + 1, T), dtype=np.float64)
    p_st = np.zeros((nr + 1, T), dtype=np.float64)
    three = np.zeros(nr + 1, dtype=bool)
    photo = np.zeros(nr + 1, dtype=bool)
    par = {f: np.zeros(nr + 1) for f in ("a", "n", "E", "a_inf", "n_inf", "E_inf")}
    flag = {f: np.zeros(nr + 1, dtype=bool) for f in ("is_forward", "has_kinf", "is_special", "is_conden",
                                                      "is_radiative", "is_ion")}
    sec_flag = {THREE_BODY_KINF: "has_kinf", SPECIAL: "is_special", CONDEN: "is_conden",
                RADIATIVE: "is_radiative"}
    Rf = {}
    for rec in records:
        i = rec["row"]
        for s, (sp, st) in enumerate(rec["reac"].items()):
            r_idx[i, s], r_st[i, s] = sp, st
            p_idx[i + 1, s], p_st[i + 1, s] = sp, st
        for s, (sp, st) in enumerate(rec["prod"].items()):
            p_idx[i, s], p_st[i, s] = sp, st
            r_idx[i + 1, s], r_st[i + 1, s] = sp, st
        three[i] = rec["m_reac"]
        three[i + 1] = rec["m_prod"]
        sec = rec["section"]
        photo[i] = sec == PHOTO
        flag["is_forward"][i] = True
        if sec in sec_flag:
            flag[sec_flag[sec]][i] = flag[sec_flag[sec]][i + 1] = True
        if sec == ION:
            flag["is_ion"][i] = True
        cols = rec["nums"]
        if sec in (TWO_BODY, THREE_BODY_KINF, THREE_BODY_NO_KINF):
            if len(cols) >= 3:
                par["a"][i], par["n"][i], par["E"][i] = cols[0], cols[1], cols[2]
            if sec == THREE_BODY_KINF and len(cols) >= 6:
                par["a_inf"][i], par["n_inf"][i], par["E_inf"][i] = cols[3], cols[4], cols[5]
        Rf[i] = rec["eq"]
    if stop_rev is None:
        stop_rev = photo_row if photo_row is not None else nr + 1
    return NetworkTables(species=tuple(order), ni=ni, nr=nr, reactant_idx=r_idx,
                         product_idx=p_idx, reactant_stoich=r_st, product_stoich=p_st,
                         is_three_body=three, is_photo=photo,
                         pho_rate_index=pho_rate_index, photo_sp=tuple(photo_sp),
                         stop_rev_indx=int(stop_rev), Rf=Rf, **par, **flag)


def parse_network(path) -> NetworkTables:
    """Parse a network file on disk."""
    with open(path) as f:
        return parse_network_text(f.read())


def _term(c: int, sp: str) -> str:
    return sp if c == 1 else f"{c}*{sp}"


def format_network(two_body, three_body=(), photo=()) -> str:
    """Write reactions in the network-file format.

    ``two_body`` / ``three_body``: sequences of ``(reactants, products)`` with
    each side a sequence of ``(stoich, species)``; three-body reactions get
    ``+ M`` on both sides. ``photo``: ``(species, branch, products)`` triples.
    Ids are the odd parser rows, as in the bundled VULCAN networks.
    """
    lines = ["# synthetic mass-action network (written by jax-vulcan_b200.network)",
             "# two-body Reactions"]
    fid = 1

    def eq(reac, prod, m=False):
        lhs = " + ".join(_term(c, s) for c, s in reac) + (" + M" if m else "")
        rhs = " + ".join(_term(c, s) for c, s in prod) + (" + M" if m else "")
        return f"{lhs} -> {rhs}"

    for reac, prod in two_body:
        lines.append(f"{fid:5d} [ {eq(reac, prod)} ]  1.0E-10  0.0  0.0")
        fid += 2
    if three_body:
        lines.append("# 3-body reactions without high-pressure rates")
        for reac, prod in three_body:
            lines.append(f"{fid:5d} [ {eq(reac, prod, True)} ]  1.0E-30  0.0  0.0")
            fid += 2
    lines.append("# reverse stops")
    if photo:
        lines.append("# photo disscoiation (no reversals)")
        for sp, br, prod in photo:
            lines.append(f"{fid:5d} [ {eq([(1, sp)], prod)} ]  {sp}  {br}")
            fid += 2
    return "\n".join(lines) + "\n"
