"""Basis-set text in the two formats basis-set libraries export, read into
the PySCF internal format this package (and the reference, through
``mol._basis``, ``OmegaQMC/psi/gto.py:896-900``) works with:
``{element: [[am, [alpha, c1, c2, ...], ...], ...]}``.

The reference gets its basis sets from PySCF's library by name
(``OmegaQMC/vmc_gto.py:217-452``); that library is not part of this
package, so users bring the text of the set they want (for example the
NWChem or Gaussian94 export of a basis-set exchange) and pass it to
:func:`omegaqmc_b200.generate_molecular_orbitals`.

* NWChem: blocks of ``<element> <shell>`` lines followed by rows of
  ``exponent c1 [c2 ...]`` (several coefficient columns = a general
  contraction), optional ``BASIS ...`` / ``END`` lines and ``#`` comments.
* Gaussian94: per element an ``<element> 0`` line, then shells
  ``<type> <nprim> <scale>`` each followed by ``nprim`` rows, elements
  separated by ``****``; Fortran ``D`` exponents are accepted.

An ``SP`` (or ``L``) shell becomes an s and a p entry sharing the exponents,
as PySCF's parsers do.  The scale factor of a Gaussian94 shell multiplies
the exponents by its square.
"""
from __future__ import annotations

import os

__all__ = ["parse_basis_text", "load_basis"]

_AM = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5, "I": 6}


def _num(tok):
    return float(tok.replace("D", "E").replace("d", "e"))


def _is_num(tok):
    try:
        _num(tok)
        return True
    except ValueError:
        return False


def _element(tok):
    s = tok.strip()
    return s[:1].upper() + s[1:].lower()


def _add(out, elem, am_label, rows):
    """Append the shell(s) of one block; rows are [exponent, c1, c2, ...]."""
    if not rows:
        raise ValueError(f"shell {am_label} of {elem} has no primitives")
    width = {len(r) for r in rows}
    if len(width) != 1 or min(width) < 2:
        raise ValueError(f"shell {am_label} of {elem}: rows of unequal or too short length")
    lab = am_label.upper()
    if lab in ("SP", "L"):
        if min(width) != 3:
            raise ValueError(f"SP shell of {elem} needs an s and a p coefficient per row")
        out.setdefault(elem, []).append([0] + [[r[0], r[1]] for r in rows])
        out.setdefault(elem, []).append([1] + [[r[0], r[2]] for r in rows])
        return
    if lab not in _AM:
        raise ValueError(f"unknown shell type {am_label!r} for {elem}")
    out.setdefault(elem, []).append([_AM[lab]] + [list(r) for r in rows])


def _parse_nwchem(lines):
    out = {}
    elem = lab = None
    rows = []
    for raw in lines:
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        toks = line.split()
        head = toks[0].upper()
        if head in ("BASIS", "END"):
            if elem is not None:
                _add(out, elem, lab, rows)
                elem, rows = None, []
            continue
        if not _is_num(toks[0]):
            if len(toks) < 2:
                raise ValueError(f"cannot read basis line {raw!r}")
            if elem is not None:
                _add(out, elem, lab, rows)
            elem, lab, rows = _element(toks[0]), toks[1], []
            continue
        if elem is None:
            raise ValueError(f"primitive before any shell header: {raw!r}")
        rows.append([_num(t) for t in toks])
    if elem is not None:
        _add(out, elem, lab, rows)
    return out


def _parse_gaussian94(lines):
    out = {}
    elem = None
    it = iter(lines)
    for raw in it:
        line = raw.split("!", 1)[0].strip()
        if not line:
            continue
        if line.startswith("****"):
            elem = None
            continue
        toks = line.split()
        if elem is None:
            elem = _element(toks[0])
            continue
        lab, nprim = toks[0], int(toks[1])
        scale = _num(toks[2]) if len(toks) > 2 else 1.0
        rows = []
        while len(rows) < nprim:
            line2 = next(it, None)
            if line2 is None:
                raise ValueError(f"shell {lab} of {elem}: {nprim} primitives announced, "
                                 f"{len(rows)} found")
            r = line2.split("!", 1)[0].split()
            if not r:
                continue
            rows.append([_num(t) for t in r])
        for r in rows:
            r[0] *= scale * scale
        _add(out, elem, lab, rows)
    return out


def parse_basis_text(text, fmt=None):
    """Basis dict from NWChem or Gaussian94 text (``fmt`` ``"nwchem"``,
    ``"gaussian94"`` or None to tell them apart by the ``****`` separators)."""
    lines = text.splitlines()
    if fmt is None:
        fmt = "gaussian94" if any(l.strip().startswith("****") for l in lines) else "nwchem"
    fmt = fmt.lower()
    if fmt == "nwchem":
        out = _parse_nwchem(lines)
    elif fmt in ("gaussian94", "g94", "gaussian"):
        out = _parse_gaussian94(lines)
    else:
        raise ValueError(f"unknown basis format {fmt!r}")
    if not out:
        raise ValueError("no basis functions found in the text")
    return out


def load_basis(spec, elements=None, fmt=None):
    """Basis dict from a dict (returned as is, or a per-element dict of
    texts), a file path or basis text; ``elements`` restricts and checks the
    elements present."""
    if isinstance(spec, dict):
        out = {}
        for el, v in spec.items():
            if isinstance(v, str):
                sub = parse_basis_text(v if "\n" in v or not os.path.exists(v)
                                       else open(v).read(), fmt)
                out[_element(el)] = sub.get(_element(el)) or next(iter(sub.values()))
            else:
                out[_element(el)] = v
    else:
        text = open(spec).read() if os.path.exists(spec) else spec
        out = parse_basis_text(text, fmt)
    if elements is not None:
        missing = sorted(set(elements) - set(out))
        if missing:
            raise ValueError(f"no basis functions for {', '.join(missing)}")
        out = {e: out[e] for e in elements}
    return out
