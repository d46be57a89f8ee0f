"""The reference's checkpoint files: ``prefix.bin`` + ``prefix_setup.txt``.

MHDSolver::save_state / load_state (src/library/mhd_solver.inlrb:1023-1050)
write the state dump and the two setup pods as text: GlobalSetup, a line of
``################``, then LocalSetup, each as a member count followed by
``name value`` lines (src/nushio_script/persistent_pod.hrb:129-176; generated
src/library/mhd_solver.h:181-232, 438-507).  Numbers are written with C++'s
default stream format (6 significant digits), strings with ``%xx`` escapes.
On load the reference keeps only generation and current_time from GlobalSetup
(and the rank, directory and shear displacement/velocity of LocalSetup).

The 6-digit current_time makes the reference's own restarts lossy.  Files
written here carry one extra GlobalSetup member, ``current_time_exact``
(17 significant digits), which the reference's reader skips (it reads the
member count and ignores names it does not know) and this reader prefers, so a
restart from a file written here continues bitwise as the uninterrupted run,
and a file written by either code loads in the other.
"""
from __future__ import annotations

import math

import numpy as np

SPACER = "################"


def _num(x) -> str:
    """std::ostream << x with the default format (precision 6, %g style)."""
    if isinstance(x, (int, np.integer)):
        return str(int(x))
    return "%.6g" % float(x)


def _enc(s: str) -> str:
    """encode_member(std::string): bytes outside 33..126 and '%' as %xx."""
    out = []
    for c in s.encode():
        out.append(chr(c) if 33 <= c <= 126 and c != ord("%") else "%%%02x" % c)
    return "".join(out)


def _dec(s: str) -> str:
    out = bytearray()
    i = 0
    while i < len(s):
        if s[i] == "%":
            out.append(int(s[i + 1:i + 3], 16))
            i += 3
        else:
            out += s[i].encode()
            i += 1
    return out.decode(errors="replace")


def shear_displacement(cfg, time: float) -> float:
    """relative_displacement()'s normalized displacement (mhd_solver.inlrb:244-259):
    the azimuthal offset of a rank's upper shearing boundary, folded into the
    box, as the reference's float (the same for every radial rank, whose
    relative velocity is that of its own slab)."""
    if cfg.problem != "shearing_box":
        return 0.0
    d = cfg.derived()
    d0 = 0.0 + time * d["relative_velocity"]
    fold = math.floor(d0 / float(d["extent_x"]))
    return float(np.float32(d0 - float(np.float32(np.float32(fold) * d["extent_x"]))))


def setup_text(cfg, generation: int, time: float, output_directory: str = ".",
               mpi_prefix: str = None, rank: int = 0) -> str:
    """The ``_setup.txt`` that the reference's save_state writes for this box
    and clock, plus the ``current_time_exact`` member.  ``rank`` is the radial
    slab's rank when ``cfg.parallel_size_y`` > 1 (ranks along Y only), else 0."""
    d = cfg.derived()
    py = max(1, cfg.parallel_size_y)
    if not 0 <= rank < py:
        raise ValueError("rank must be in [0, parallel_size_y)")
    if mpi_prefix is None:
        mpi_prefix = "%04d" % rank
    local = (cfg.size_x, cfg.size_y - 2 * cfg.margin_y, cfg.size_z - 2 * cfg.margin_z)
    gsize = (local[0], py * local[1], local[2])
    psize = (1, py, 1)
    rank3 = (0, rank, 0)
    gext = (np.float32(cfg.extent_x), np.float32(cfg.extent_y), np.float32(cfg.extent_z))
    sizes = (cfg.size_x, cfg.size_y, cfg.size_z)
    margins = (0, cfg.margin_y, cfg.margin_z)
    dd = (d["dx"], d["dy"], d["dz"])
    g = [("generation", generation), ("real_size", 4), ("real_precision", "float"),
         ("current_time", float(time)), ("parallel_size", py)]
    for k, ax in enumerate("xyz"):
        g += [("global_size_" + ax, gsize[k]), ("parallel_size_" + ax, psize[k]),
              ("global_extent_" + ax, gext[k]), ("global_corner_" + ax, 0.0), ("d" + ax.upper(), dd[k])]
    rel_vel = d["relative_velocity"] if cfg.problem == "shearing_box" else 0.0
    loc = [("mpi_rank", rank), ("output_directory", output_directory), ("mpi_prefix", mpi_prefix),
           ("relative_displacement", shear_displacement(cfg, time)), ("relative_velocity", rel_vel),
           ("computational_size", cfg.cells)]
    for k, ax in enumerate("xyz"):
        # LocalSetup: kGlobalCorner + (kLocalSize * rank - kMarginSize) * kD (mhd_solver.h:311-317)
        corner = np.float32(np.float32(local[k] * rank3[k] - margins[k]) * dd[k])
        loc += [("computational_size_" + ax, sizes[k]), ("margin_" + ax, margins[k]),
                ("computational_corner_" + ax, corner), ("computational_extent_" + ax, d["extent_" + ax]),
                ("d" + ax.upper(), dd[k])]

    def pod(members):
        lines = [str(len(members))]
        for name, v in members:
            lines.append(f"{name} {_enc(v) if isinstance(v, str) else _num(v)}")
        return "\n".join(lines) + "\n"
    glob = pod(g + [("current_time_exact", 0.0)])
    glob = glob.replace("current_time_exact 0\n", "current_time_exact %.17g\n" % float(time))
    return glob + "\n" + SPACER + "\n" + pod(loc) + "\n"


def parse_setup(text: str):
    """(GlobalSetup members, LocalSetup members) as dicts of strings, read the
    way the reference's operator>> reads them: a count, that many name/value
    tokens, the spacer token, then the second pod."""
    tok = text.split()
    i = 0

    def pod():
        nonlocal i
        n = int(tok[i])
        i += 1
        m = {}
        for _ in range(n):
            m[tok[i]] = tok[i + 1]
            i += 2
        return m
    glob = pod()
    i += 1  # SPACER
    loc = pod() if i < len(tok) else {}
    return glob, loc


def clock_from_setup(text: str):
    """(generation, current_time) as load_state restores them; the exact time
    when the file carries it."""
    glob, _ = parse_setup(text)
    t = glob.get("current_time_exact", glob["current_time"])
    return int(glob["generation"]), float(t)


def directory_of(text: str) -> str:
    """LocalSetup's output_directory of a setup file."""
    return _dec(parse_setup(text)[1].get("output_directory", ""))
