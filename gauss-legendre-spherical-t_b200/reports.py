"""Run reports in the reference driver's text layout.

The reference's driver (test/full_example.cu:94-101, :213-233) and its
utilities (utils/utils.cpp:60-168) print a run as: a ``BENCH_INPUT`` line,
the set-up summary of ``glst_force::init`` (src/glst_force.cu:245-293),
per-phase mean and standard deviation over the iterations, the direct
Coulomb runtime and an error report against direct Coulomb.  Its
``utils/parse_glst_results.py`` turns such logs into one CSV.  The functions
here produce the same layout from this package's results, so runs of this
engine and of the reference can be put side by side with that script.
"""
import math

import numpy as np

PHASE_LABELS = (
    ("assign", "                   Assign atoms to cells"),
    ("structure_factors", "             Calculate structure factors"),
    ("shell_sums", "            Sum remote structure factors"),
    ("long_range", "  Calculate long-range energy and forces"),
    ("near_field", " Calculate short-range energy and forces"),
    ("combine", "         Communicate energies and forces"),
)


def error_stats(glst, coul):
    """Per component (fx, fy, fz, en): min, max and mean of the absolute
    error, RMS error, each also divided by the RMS of the GLST value
    (utils/utils.cpp:60-125; error = Coulomb - GLST)."""
    out = {}
    for name, g, c in zip(("fx", "fy", "fz", "en"), glst, coul):
        g = np.asarray(g, dtype=np.float64)
        c = np.asarray(c, dtype=np.float64)
        err = c - g
        a = np.abs(err)
        rms_g = math.sqrt(float(np.mean(g * g)))
        st = {"min": float(a.min()), "max": float(a.max()), "avg": float(a.mean()),
              "rms": math.sqrt(float(np.mean(err * err)))}
        out[name] = {k: (v, v / rms_g if rms_g else float("inf")) for k, v in st.items()}
    return out


def _sci(v, sign=True):
    # C++ std::scientific (6 digits), with std::showpos where the reference sets it
    return ("%+.6e" if sign else "%.6e") % v


def format_error_report(stats, tol):
    lines = ["", "Target error: " + _sci(tol, sign=False), ""]
    titles = (("fx", "  X Force Error: "), ("fy", "  Y Force Error: "), ("fz", "  Z Force Error: "),
              ("en", "   Energy Error: "))
    labels = (("min", "         Absolute Min: "), ("max", "         Absolute Max: "),
              ("avg", "              Average: "), ("rms", "    Root Mean Squared: "))
    for comp, title in titles:
        lines.append(title)
        for key, label in labels:
            v, n = stats[comp][key]
            lines.append("%s%s (Norm: %s)" % (label, _sci(v), _sci(n)))
        lines.append("")
    return "\n".join(lines) + "\n"


def format_setup(info, box):
    """The set-up summary glst_force::init prints (one GPU)."""
    n = list(info.ncell)
    l = info.cell_dim
    g = lambda v: "%g" % v
    lines = ["",
             "          Number of atoms: %d" % info.natom,
             "    System dimensions [A]: %s x %s x %s" % tuple(g(b) for b in box),
             "          Number of cells: %d, %d, %d" % tuple(n),
             "      Cell dimensions [A]: %s x %s x %s" % (g(l), g(l), g(l)),
             "  Total space covered [A]: %s x %s x %s" % tuple(g(k * l) for k in n),
             "           Number of GPUs: 1",
             "",
             "  Number of alpha groups: %d" % info.ngroup,
             "       Total number of cubature nodes: %d" % info.num_nodes]
    for i in range(min(info.ngroup, 16)):
        lines.append("  Number of cubature nodes in group %d: %d" % (i, info.group_nodes[i]))
    lines.append("  Number of cubature nodes per device: ~%d" % info.num_nodes)
    return "\n".join(lines) + "\n"


def _mean_std(xs):
    xs = [float(x) for x in xs]
    m = sum(xs) / len(xs)
    var = sum((x - m) ** 2 for x in xs) / len(xs)
    return m, math.sqrt(var)


def format_run_log(meta, info, box, phase_ms, coulomb_ms, stats, tol):
    """The whole log.  meta: BENCH_INPUT fields (sweep, sys, tol, box_dim,
    cut, requested_gpus); phase_ms: {phase: [ms per iteration]} with the keys
    of PHASE_LABELS (missing phases print as 0); the long-range runtime is
    assignment through the long-range gather, the total all phases, per
    iteration, as the reference's driver sums them."""
    head = "BENCH_INPUT " + " ".join("%s=%s" % (k, meta[k]) for k in
                                     ("sweep", "sys", "tol", "box_dim", "cut", "requested_gpus"))
    iters = len(next(iter(phase_ms.values())))
    per = {k: list(phase_ms.get(k, [0.0] * iters)) for k, _ in PHASE_LABELS}
    lr_total = [sum(per[k][i] for k in ("assign", "structure_factors", "shell_sums", "long_range"))
                for i in range(iters)]
    total = [sum(per[k][i] for k, _ in PHASE_LABELS) for i in range(iters)]
    lines = [head, format_setup(info, box), "", "Finished %d calculations" % iters, ""]
    for k, label in PHASE_LABELS:
        m, s = _mean_std(per[k])
        lines.append("%s: %g ms (+/- %g ms)" % (label, m, s))
    lines.append("-" * 74)
    for label, xs in (("                 Long-Range GLST Runtime", lr_total),
                      ("                      Total GLST Runtime", total)):
        m, s = _mean_std(xs)
        lines.append("%s: %g ms (+/- %g ms)" % (label, m, s))
    lines += ["", "Coulomb Runtime: %g ms" % coulomb_ms]
    return "\n".join(lines) + "\n" + format_error_report(stats, tol)
