"""MPS files for the reader's parity tests: random LPs written in free or
fixed format with the features the reader handles (objective constant, every
RANGES and BOUNDS form, integer markers, duplicate coefficients, comments) and
numbers in many notations, including ones long enough to need the library
fallback of the digit parser."""
import numpy as np

FORMS = ("repr", "e6", "g17", "D", "plus", "trail_dot", "lead_dot", "long")


def number(v, rng, fixed):
    form = FORMS[int(rng.integers(0, 3 if fixed else len(FORMS)))]
    if form == "repr":
        s = repr(float(v))
    elif form == "e6":
        s = f"{v:.6e}"
    elif form == "g17":
        s = f"{v:.17g}"
    elif form == "D":
        s = f"{v:.5E}".replace("E", "D")
    elif form == "plus":
        s = ("+" if v >= 0 else "") + f"{v:.9g}"
    elif form == "trail_dot":
        s = f"{round(v):d}."
    elif form == "lead_dot":
        frac = f"{abs(v) % 1:.7f}"[1:] if abs(v) % 1 else ".5"
        s = ("-" if v < 0 else "") + frac
    else:
        s = f"{v:.25f}"
    if fixed and len(s) > 12:
        s = f"{v:.5g}"
    return s


def write_mps(rng, m=12, n=20, fixed=False):
    names_r = [f"R{i:04d}" for i in range(m)]
    names_c = [f"C{j:04d}" for j in range(n)]
    types = rng.choice(list("ELG"), size=m)
    lines = ["* generated for the reader parity tests", f"NAME          case{int(rng.integers(1000))}", "ROWS",
             " N  OBJ"]
    if rng.random() < 0.3:
        lines.append(" N  FREEROW")
    lines += [f" {t}  {r}" for t, r in zip(types, names_r)]
    lines.append("COLUMNS")
    marked = set(rng.choice(n, size=3, replace=False).tolist())
    in_marker = False
    for j in range(n):
        if (j in marked) != in_marker:
            lines.append("    MARKER    'MARKER'                 " + ("'INTORG'" if not in_marker else "'INTEND'"))
            in_marker = not in_marker
        rows = sorted(rng.choice(m, size=int(rng.integers(1, 5)), replace=False).tolist())
        if rng.random() < 0.2:
            rows.append(rows[0])          # a duplicate coefficient
        cells = []
        if rng.random() < 0.8:
            cells.append(("OBJ", rng.uniform(-5, 5)))
        cells += [(names_r[i], rng.uniform(-10, 10)) for i in rng.permutation(rows)]
        for k in range(0, len(cells), 2):
            pair = cells[k:k + 2]
            if fixed:
                line = f"    {names_c[j]:<8}  {pair[0][0]:<8}  {number(pair[0][1], rng, True):>12}"
                if len(pair) > 1:
                    line += f"   {pair[1][0]:<8}  {number(pair[1][1], rng, True):>12}"
            else:
                line = f"    {names_c[j]}  " + "  ".join(f"{r} {number(v, rng, False)}" for r, v in pair)
            lines.append(line)
            if rng.random() < 0.05:
                lines.append("* a comment between cards")
    if in_marker:
        lines.append("    MARKER    'MARKER'                 'INTEND'")
    lines.append("RHS")
    cells = [(r, rng.uniform(-20, 20)) for r in names_r if rng.random() < 0.7]
    if rng.random() < 0.5:
        cells.append(("OBJ", rng.uniform(-3, 3)))
    for k in range(0, len(cells), 2):
        pair = cells[k:k + 2]
        if fixed:
            line = f"    {'RHS':<8}  {pair[0][0]:<8}  {number(pair[0][1], rng, True):>12}"
            if len(pair) > 1:
                line += f"   {pair[1][0]:<8}  {number(pair[1][1], rng, True):>12}"
        else:
            line = "    RHS  " + "  ".join(f"{r} {number(v, rng, False)}" for r, v in pair)
        lines.append(line)
    if rng.random() < 0.2 and not fixed:
        lines.append("    RHS2  " + f"{names_r[0]} 99.0")       # a second set: ignored
    if rng.random() < 0.8:
        lines.append("RANGES")
        for r in names_r:
            if rng.random() < 0.4:
                v = rng.uniform(-6, 6)
                lines.append(f"    {'RNG':<8}  {r:<8}  {number(v, rng, True):>12}" if fixed
                             else f"    RNG  {r} {number(v, rng, False)}")
    lines.append("BOUNDS")
    for j in range(n):
        kind = rng.choice(["none", "LO", "UP", "UPneg", "FX", "FR", "MI", "PL", "BV", "LI", "UI", "LOUP"])
        c = names_c[j]
        val = lambda lo, hi: number(rng.uniform(lo, hi), rng, fixed)
        entries = []
        if kind == "LO":
            entries = [("LO", val(-5, 5))]
        elif kind == "UP":
            entries = [("UP", val(0, 50))]
        elif kind == "UPneg":
            entries = [("UP", val(-5, -0.5))]
        elif kind == "FX":
            entries = [("FX", val(-2, 2))]
        elif kind in ("FR", "MI", "PL", "BV"):
            entries = [(kind, None)]
        elif kind == "LI":
            entries = [("LI", val(-3, 3))]
        elif kind == "UI":
            entries = [("UI", val(1, 9))]
        elif kind == "LOUP":
            entries = [("LO", val(-5, 0)), ("UP", val(1, 9))]
        for t, v in entries:
            if fixed:
                lines.append(f" {t:<2} {'BND':<8}  {c:<8}" + (f"  {v:>12}" if v is not None else ""))
            else:
                lines.append(f" {t} BND {c}" + (f" {v}" if v is not None else ""))
    lines.append("ENDATA")
    return "\n".join(lines) + "\n"


def lp_to_mps(lp, name="planted"):
    """Free-format MPS text of a host LP (row sides as E/L/G plus RANGES for
    two-sided rows; LO/UP/FX/FR/MI bounds); values written with repr.  A free
    row is written as an L row with right-hand side 1e9, which no feasible
    point of these models reaches."""
    rows = [f"R{i}" for i in range(lp.m)]
    lines = [f"NAME {name}", "ROWS", " N OBJ"]
    kinds = []
    for i in range(lp.m):
        lo, hi = lp.AL[i], lp.AU[i]
        k = "E" if lo == hi else "L" if np.isneginf(lo) else "G"
        kinds.append(k)
        lines.append(f" {k} {rows[i]}")
    lines.append("COLUMNS")
    lp = lp.ensure_transpose()
    ptr, idx = lp.at_ptr, lp.at_idx
    for j in range(lp.n):
        cells = [("OBJ", lp.c[j])] if lp.c[j] != 0.0 else []
        cells += [(rows[idx[q]], lp.at_val[q]) for q in range(ptr[j], ptr[j + 1])]
        if not cells:
            cells = [("OBJ", 0.0)]
        for r, v in cells:
            lines.append(f"    C{j} {r} {float(v)!r}")
    lines.append("RHS")
    for i, k in enumerate(kinds):
        side = lp.AU[i] if k == "L" else lp.AL[i]
        if np.isposinf(side):
            side = 1.0e9
        if side != 0.0:
            lines.append(f"    RHS {rows[i]} {float(side)!r}")
    lines.append("RANGES")
    for i, k in enumerate(kinds):
        if k == "G" and np.isfinite(lp.AU[i]):
            lines.append(f"    RNG {rows[i]} {float(lp.AU[i] - lp.AL[i])!r}")
    lines.append("BOUNDS")
    for j in range(lp.n):
        lo, hi = lp.l[j], lp.u[j]
        if lo == hi:
            lines.append(f" FX BND C{j} {float(lo)!r}")
            continue
        if np.isneginf(lo) and np.isposinf(hi):
            lines.append(f" FR BND C{j}")
            continue
        if np.isneginf(lo):
            lines.append(f" MI BND C{j}")
        elif lo != 0.0:
            lines.append(f" LO BND C{j} {float(lo)!r}")
        if np.isfinite(hi):
            lines.append(f" UP BND C{j} {float(hi)!r}")
    lines.append("ENDATA")
    return "\n".join(lines) + "\n"


# Inputs the reader must reject (both readers fail on each).
BAD = {
    "unknown_row": "NAME x\nROWS\n N OBJ\n L R1\nCOLUMNS\n    X1 OBJ 1.0 R9 2.0\nENDATA\n",
    "maximise": "NAME x\nOBJSENSE\n    MAX\nROWS\n N OBJ\n L R1\nCOLUMNS\n    X1 OBJ 1.0 R1 2.0\nENDATA\n",
    "quadratic": "NAME x\nROWS\n N OBJ\n L R1\nCOLUMNS\n    X1 OBJ 1.0 R1 2.0\nQUADOBJ\n    X1 X1 1.0\nENDATA\n",
    "bad_bound": "NAME x\nROWS\n N OBJ\n L R1\nCOLUMNS\n    X1 OBJ 1.0 R1 2.0\nBOUNDS\n SC BND X1 3.0\nENDATA\n",
    "empty": "NAME x\nENDATA\n",
}
