"""Run summary CSV and conservation checks, the host-side counterpart of the reference's
complab_diag::Diagnostics (src/complab3d_diagnostics.hh): one row per diagnostic interval with the
iteration, porosity and open-voxel count and, for every substrate and microbe, its total, mean,
minimum, maximum and `held` mass; named sums (<conserve>Fe2+FeS</conserve>) checked against their
first value with the relative drift |sum - first| / max(|first|, |sum|); a warning the first time
a check drifts past the tolerance or a field goes below -1e-9; a final report with a PASS / FAIL /
SKIPPED verdict per check. The CSV, the messages and the report have the reference's format, so
its post-processing reads them unchanged.

row_from_domain() fills a row from the library's reductions (clb_reduce): totals, minima and
maxima over the open voxels of x = 1..nx-2, `held` = the whole lattice's population content
minus that total (the mass at walls, in the boundary planes and in flight on wall links), so
total + held is the lattice's whole content, the quantity the conservation checks compare.
"""
from __future__ import annotations


class FieldStat:
    def __init__(self, name, total=0.0, mean=0.0, minv=0.0, maxv=0.0, held=0.0):
        self.name, self.total, self.mean, self.minv, self.maxv, self.held = name, total, mean, minv, maxv, held

    def conserved(self):
        return self.total + self.held


class Row:
    def __init__(self, iteration=0, porosity=0.0, open_voxels=0, fields=()):
        self.iteration, self.porosity, self.open_voxels = int(iteration), float(porosity), int(open_voxels)
        self.fields = list(fields)


def _split_plus(expr):
    return [t.replace(" ", "").replace("\t", "") for t in expr.split("+") if t.replace(" ", "").replace("\t", "")]


def _g(x):
    return "%.17g" % x


def _e(x, digits):
    return "%.*e" % (digits, x)


class _Check:
    def __init__(self, expr):
        self.expr, self.terms = expr, _split_plus(expr)
        self.first, self.have_first, self.comparisons = 0.0, False, 0
        self.worst, self.warned, self.skipped = 0.0, False, False


class Diagnostics:
    """complab_diag::Diagnostics: configure(), add_conserve(), record(row) -> message,
    final_report() -> text."""

    def __init__(self):
        self.enabled, self.path, self.tol, self.master = False, "", 1e-6, True
        self.rows, self.any_fail, self.checks, self.neg_warned = 0, False, [], []

    def configure(self, enabled, path, tol, is_master=True):
        self.enabled, self.path, self.tol, self.master = bool(enabled), str(path), float(tol), bool(is_master)

    def add_conserve(self, expr):
        c = _Check(expr)
        if c.terms:
            self.checks.append(c)

    def failed(self):
        return self.any_fail

    def record(self, r: Row) -> str:
        if not self.enabled:
            return ""
        msg = ""
        if self.master:
            if self.rows == 0:
                self._write_header(r)
            self._write_row(r)
        self.rows += 1
        for k in self.checks:
            total, complete = 0.0, True
            for t in k.terms:
                f = next((f for f in r.fields if f.name == t), None)
                if f is None:
                    complete = False
                    break
                total += f.conserved()
            if not complete:
                if not k.warned:
                    k.warned = k.skipped = True
                    msg += ("  [DIAG] <conserve>" + k.expr + "</conserve> names a substrate that "
                            "does not exist; the check is skipped.\n")
                continue
            if not k.have_first:
                k.first, k.have_first = total, True
                continue
            scale = max(abs(k.first), abs(total), 1e-300)
            drift = abs(total - k.first) / scale
            k.comparisons += 1
            k.worst = max(k.worst, drift)
            if drift > self.tol and not k.warned:
                k.warned, self.any_fail = True, True
                msg += ("  [DIAG] MASS BALANCE: %s drifted %s (tolerance %s) by step %d.\n"
                        "  [DIAG]   started %s, now %s.\n" % (k.expr, _e(drift, 3), _e(self.tol, 1), r.iteration,
                                                             "%.10g" % k.first, "%.10g" % total))
                msg += ("  [DIAG]   An inlet held at a fixed value, an unbalanced reaction or too long a\n"
                        "  [DIAG]   time step for the rates are the usual causes.\n")
        for f in r.fields:
            if f.minv < -1e-9 and f.name not in self.neg_warned:
                self.neg_warned.append(f.name)
                self.any_fail = True
                msg += "  [DIAG] %s went negative (%s) at step %d.\n" % (f.name, _e(f.minv, 3), r.iteration)
        return msg

    def final_report(self) -> str:
        if not self.enabled:
            return ""
        s = "\n  [DIAG] summary written to " + self.path + "\n"
        for k in self.checks:
            if k.skipped:
                verdict = "SKIPPED (unknown substrate)"
            elif k.comparisons == 0:
                verdict = ("SKIPPED (never compared: fewer than two diagnostic rows, so there was no "
                           "baseline to compare against)")
            else:
                verdict = "PASS" if k.worst <= self.tol else "FAIL"
            s += "  [DIAG] %-24s worst relative drift %s  %s\n" % (k.expr, _e(k.worst, 3), verdict)
        ran = sum(1 for k in self.checks if not k.skipped and k.comparisons > 0)
        if self.checks:
            if ran == 0:
                s += ("  [DIAG] verdict: NOT CHECKED -- no check compared two rows; record at least two "
                      "rows.\n")
            else:
                s += "  [DIAG] verdict: " + ("FAIL" if self.any_fail else "PASS") + "\n"
        return s

    def _write_header(self, r):
        with open(self.path, "w") as f:
            f.write("# run summary, one row per diagnostic interval (clb)\n")
            f.write("# totals, minima and maxima over the open voxels of x=1..nx-2; means divided by the\n")
            f.write("# open voxel count of the live mask; <name>_held = the whole lattice's content minus\n")
            f.write("# the total, so _total + _held is what the conservation checks compare.\n")
            f.write("iteration,porosity,open_voxels")
            for fs in r.fields:
                n = fs.name
                f.write(",%s_total,%s_mean,%s_min,%s_max,%s_held" % (n, n, n, n, n))
            f.write("\n")

    def _write_row(self, r):
        # reopened per row: a run that is killed still leaves a complete CSV
        with open(self.path, "a") as f:
            f.write("%d,%s,%d" % (r.iteration, _g(r.porosity), r.open_voxels))
            for fs in r.fields:
                f.write("," + ",".join(_g(v) for v in (fs.total, fs.mean, fs.minv, fs.maxv, fs.held)))
            f.write("\n")


def row_from_domain(D, iteration, substrate_names, microbe_names=()):
    """One row from the domain's reductions (clb_reduce): substrates' totals, minima and maxima
    over the open voxels of x = 1..nx-2, held = whole-lattice content - total; microbes' totals
    (held 0: the biomass fields hold no populations)."""
    st = D.reduce()
    nx, ny, nz = D.nx, D.ny, D.nz
    opened = int(st["open_voxels"])
    vox = (nx - 2) * ny * nz
    fields = []
    for s, name in enumerate(substrate_names):
        tot = float(st["total"][s])
        fields.append(FieldStat(name, tot, tot / opened if opened else 0.0, float(st["min"][s]), float(st["max"][s]),
                                float(st["content"][s]) - tot))
    for m, name in enumerate(microbe_names):
        b = D.biomass(m).reshape(nx, ny, nz)[1:-1]
        tot = float(st["biomass"][m])
        fields.append(FieldStat(name, tot, tot / opened if opened else 0.0, float(b.min()), float(b.max()), 0.0))
    return Row(iteration, opened / vox if vox else 0.0, opened, fields)
