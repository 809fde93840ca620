"""Measurement output in the reference's file formats.

`spec_NNNN.txt` follows Spectrum::write (src/spectrum/spectrum.cxx:167-183) and
the file name of measure() (src/meas.cxx:41-44): a `# a: <a>` line, a column
header, then `k P(k) count` per non-empty shell in C++ `std::scientific` form,
so the reference's scripts/plot_spectrum.py reads the files unchanged.
"""
from __future__ import annotations

import os


def format_spectrum(a: float, k, P, count) -> str:
    """Text of a spectrum file (shells with count 0 are skipped)."""
    lines = [f"# a: {a:g}", "# k_phys      P(k)          count"]
    for kk, pp, cc in zip(k, P, count):
        if int(cc) == 0:
            continue
        lines.append(f"{float(kk):.6e}  {float(pp):.6e}  {int(cc)}")
    return "\n".join(lines) + "\n"


def write_spectrum(field, directory: str, meas_number: int, source: int = 0) -> str:
    """Write the reference-shell spectrum of |psi|^2 (source 0) or V (1) of a
    Field as <directory>/spec_<meas_number:04d>.txt; returns the path."""
    from . import SPEC_REFERENCE
    k, P, c = field.spectrum(source, SPEC_REFERENCE)
    path = os.path.join(directory, f"spec_{meas_number:04d}.txt")
    with open(path, "w") as fh:
        fh.write(format_spectrum(field.a(), k, P, c))
    return path


def format_profile(rows) -> str:
    """A profile summary in the spirit of the reference's profile.log
    (src/profiler.h:82-154): one line per timed section, `name  total_ms
    calls  ms_per_call  share`, from (name, total_ms, calls) rows."""
    tot = sum(r[1] for r in rows) or 1.0
    out = [f"{'section':28s} {'total_ms':>12s} {'calls':>8s} {'ms/call':>12s} {'share':>7s}"]
    for name, ms, calls in rows:
        out.append(f"{name:28s} {ms:12.3f} {calls:8d} {ms / max(calls, 1):12.5f} {100.0 * ms / tot:6.1f}%")
    return "\n".join(out) + "\n"
