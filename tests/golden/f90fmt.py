"""Fortran formatted output for the interpreted reference programs (f90py).

Test infrastructure only: renders the `write` statements of the reference's
Tecplot writer (output_ASCII, natural-convection_2dim_mono.f90:818-843 and
natural-convection_3dim_mono.f90:1097-1121) the way gfortran does, so the
text the reference program writes becomes a fixture.  It is written from the
Fortran standard's rules for the edit descriptors those programs use, apart
from and without reference to the library's own writer:

  nX          n blanks
  'text'      the text
  Iw          the integer right-justified in w columns
  Ew.d        [-]0.d1...dd E+xx, d significant digits correctly rounded,
              right-justified in w columns (exponent digits: E+xx for
              |exp| <= 99, +xxx up to 999), asterisks if it does not fit
  r( ... )    the group r times
A record ends at the first data descriptor left without an item (the
character descriptors before it are still written).  List-directed output of
character items (`write(u,*) 'text'`) writes one blank, then the items.
"""
from __future__ import annotations

import re
from decimal import ROUND_HALF_EVEN, Decimal


def parse_format(text: str):
    """'(1x,2(e11.4,' '),...)' -> a list of descriptors: ('x', n),
    ('lit', s), ('i', w), ('e', w, d), ('group', r, [...])."""
    text = text.strip()
    assert text[0] == "(" and text[-1] == ")", text
    items, pos = _parse_list(text, 1)
    assert pos == len(text) - 1, (text, pos)
    return items


def _parse_list(s, pos):
    items = []
    while pos < len(s):
        c = s[pos]
        if c in " ,":
            pos += 1
            continue
        if c == ")":
            return items, pos
        if c in "'\"":
            end = s.index(c, pos + 1)
            items.append(("lit", s[pos + 1:end]))
            pos = end + 1
            continue
        m = re.compile(r"(\d*)\s*\(").match(s, pos)
        if m:
            reps = int(m.group(1) or 1)
            sub, p2 = _parse_list(s, m.end())
            items.append(("group", reps, sub))
            pos = p2 + 1
            continue
        m = re.compile(r"(\d*)x", re.I).match(s, pos)
        if m:
            items.append(("x", int(m.group(1) or 1)))
            pos = m.end()
            continue
        m = re.compile(r"(\d*)e(\d+)\.(\d+)", re.I).match(s, pos)
        if m:
            for _ in range(int(m.group(1) or 1)):
                items.append(("e", int(m.group(2)), int(m.group(3))))
            pos = m.end()
            continue
        m = re.compile(r"(\d*)i(\d+)", re.I).match(s, pos)
        if m:
            for _ in range(int(m.group(1) or 1)):
                items.append(("i", int(m.group(2))))
            pos = m.end()
            continue
        raise ValueError(f"unsupported format at {s[pos:]!r}")
    raise ValueError("unbalanced format")


def edit_e(v: float, w: int, d: int) -> str:
    """Ew.d of a double."""
    v = float(v)
    neg = v < 0 or (v == 0.0 and str(v).startswith("-"))
    x = Decimal(abs(v))
    if x == 0:
        digits, exp = "0" * d, 0
    else:
        exp = x.adjusted() + 1                       # x = 0.ddd.. x 10^exp
        q = (x.scaleb(-exp)).quantize(Decimal(1).scaleb(-d), rounding=ROUND_HALF_EVEN)
        if q >= 1:                                   # rounded up to 1.000...
            exp += 1
            q = (x.scaleb(-exp)).quantize(Decimal(1).scaleb(-d), rounding=ROUND_HALF_EVEN)
        digits = format(q, f".{d}f").split(".")[1]
    if abs(exp) <= 99:
        ex = "E" + ("+" if exp >= 0 else "-") + f"{abs(exp):02d}"
    elif abs(exp) <= 999:
        ex = ("+" if exp >= 0 else "-") + f"{abs(exp):03d}"
    else:
        return "*" * w
    body = "0." + digits + ex
    s = ("-" if neg else "") + body
    if len(s) > w:
        s = ("-" if neg else "") + body[1:]          # the optional leading zero goes first
    if len(s) > w:
        return "*" * w
    return s.rjust(w)


def render(fmt_text: str, values) -> str:
    """One formatted write: the record as text, ending in a newline."""
    items = parse_format(fmt_text)
    vals = list(values)
    out = []

    def walk(seq):
        for it in seq:
            kind = it[0]
            if kind == "group":
                for _ in range(it[1]):
                    if walk(it[2]):
                        return True
            elif kind == "x":
                out.append(" " * it[1])
            elif kind == "lit":
                out.append(it[1])
            else:
                if not vals:
                    return True
                v = vals.pop(0)
                if kind == "i":
                    s = str(int(v))
                    out.append(s.rjust(it[1]) if len(s) <= it[1] else "*" * it[1])
                else:
                    out.append(edit_e(v, it[1], it[2]))
        return False

    ended = walk(items)
    if not ended and vals:
        raise NotImplementedError("format reversion is not needed by these programs")
    return "".join(out) + "\n"


def fio_open(S, unit):
    if not hasattr(S, "_io"):
        S._io = {}
    S._io[unit] = []


def fio_write_list(S, unit, vals):
    S._io[unit].append(" " + "".join(str(v) for v in vals) + "\n")


def fio_write_fmt(S, unit, fmt_text, vals):
    S._io[unit].append(render(fmt_text, vals))
