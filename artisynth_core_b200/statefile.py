"""ArtiSynth print-state files: trajectories of the engine's models in the
format the reference's regression runs record, and the reference's
comparison of two such files.

File format (MechSystemBase.writePrintStateHeader / printState,
MechSystemBase.java:1152-1225): a sequence of sections

    TEST "description"
    comps: [ P P F R4 ]
    t=0.0:
    v: <velocity state of the active dynamic components>
    x: <position state of the active dynamic components>
    t=0.01:
    ...

'P' is a particle (3 velocity and 3 position values: every active FEM node),
'F' a frame (6 velocity values, 7 position values: position and unit
quaternion), 'R<n>' the n reduced coordinates that follow a frame.  Times are
written as Java's Double.toString; the state values with the format the
regression scripts select (femRegressionTest.py: setPrintState("%g")).

compare_files() restates CompareStateFiles (CompareStateFiles.java): for each
section, pairs of files must agree in description, components and times; per
component class (point, angular, reduced) the largest norm of the difference
of a component's sub-vector over all times is normalised by the largest norm
of that sub-vector in either file (frame orientations: the rotation angle
between the quaternions over pi, magnitude 1); the section's velocity and
position errors are the largest normalised errors over the classes, and the
result is their maximum over all sections.
"""
from __future__ import annotations

import math
import re
import sys
from dataclasses import dataclass, field

import numpy as np


def java_double(d: float) -> str:
    """Double.toString: plain decimal for 1e-3 <= |d| < 1e7 (at least one
    fractional digit), computerized scientific notation otherwise, with the
    shortest digits that round-trip."""
    d = float(d)
    if d == 0.0:
        return "-0.0" if math.copysign(1.0, d) < 0 else "0.0"
    if math.isnan(d):
        return "NaN"
    if math.isinf(d):
        return "Infinity" if d > 0 else "-Infinity"
    a = abs(d)
    if 1e-3 <= a < 1e7:
        s = repr(d)
        if "e" in s or "E" in s:
            s = format(d, "f")
        return s if "." in s else s + ".0"
    mant, exp = f"{d:.17e}".split("e")
    # shortest mantissa that round-trips
    for nd in range(1, 18):
        m = f"{d:.{nd - 1}e}"
        if float(m) == d:
            mant, exp = m.split("e")
            break
    if "." not in mant:
        mant += ".0"
    return f"{mant}E{int(exp)}"


class StateWriter:
    """Writes print-state sections (file object or path)."""

    def __init__(self, out, fmt: str = "%g"):
        self._own = isinstance(out, str)
        self.f = open(out, "w") if self._own else out
        self.fmt = fmt

    def header(self, description: str, comps):
        """comps: a count of particles, or a sequence of symbols ('P', 'F',
        'R<n>')."""
        if isinstance(comps, int):
            comps = ["P"] * comps
        self.f.write('TEST "%s"\n' % description)
        self.f.write("comps: [" + "".join(" " + c for c in comps) + " ]\n")

    def state(self, t: float, v, x):
        v = np.asarray(v, dtype=np.float64).reshape(-1)
        x = np.asarray(x, dtype=np.float64).reshape(-1)
        self.f.write("t=%s:\n" % java_double(t))
        self.f.write("v: " + " ".join(self.fmt % e for e in v) + "\n")
        self.f.write("x: " + " ".join(self.fmt % e for e in x) + "\n")

    def close(self):
        if self._own:
            self.f.close()
        else:
            self.f.flush()


def write_model_trajectory(writer: StateWriter, description: str, model, solver, h: float, nsteps: int,
                           t0: float = 0.0):
    """Record a FemModel3d stepped by its MechSystemSolver: the state at t0
    and after every step, active (not fixed) nodes in node order -- the
    dynamic components of a MechModel holding one FEM model."""
    active = np.where(np.asarray(model.fixed).reshape(-1) == 0)[0]
    writer.header(description, int(active.size))
    x, v = model.getState()
    writer.state(t0, v[active], x[active])
    t = t0
    for _ in range(nsteps):
        solver.backwardEuler(h, 1)
        t += h
        x, v = model.getState()
        writer.state(t, v[active], x[active])


@dataclass
class Section:
    description: str
    comps: list
    times: list = field(default_factory=list)
    vel: list = field(default_factory=list)
    pos: list = field(default_factory=list)


_TOKEN = re.compile(r'"[^"]*"|[\[\]:=]|[^\s\[\]:=]+')


def _sizes(sym: str):
    if sym == "P":
        return 3, 3
    if sym == "F":
        return 6, 7
    if sym.startswith("R"):
        n = int(sym[1:])
        return n, n
    raise ValueError("unexpected component symbol " + sym)


def read_file(path: str):
    """Sections of a print-state file."""
    toks = _TOKEN.findall(open(path).read().replace("\r", " "))
    i, out = 0, []

    def expect(s):
        nonlocal i
        if i >= len(toks) or toks[i] != s:
            raise ValueError(f"{path}: expected {s!r} at token {i}, got {toks[i] if i < len(toks) else 'EOF'!r}")
        i += 1

    def number_run():
        nonlocal i
        vals = []
        while i < len(toks):
            try:
                vals.append(float(toks[i]))
            except ValueError:
                break
            i += 1
        return np.array(vals)

    while i < len(toks):
        expect("TEST")
        desc = toks[i].strip('"')
        i += 1
        expect("comps")
        expect(":")
        expect("[")
        comps = []
        while toks[i] != "]":
            comps.append(toks[i])
            i += 1
        i += 1
        sec = Section(desc, comps)
        nv = sum(_sizes(c)[0] for c in comps)
        npos = sum(_sizes(c)[1] for c in comps)
        while i < len(toks) and toks[i] == "t":
            expect("t")
            expect("=")
            t = float(toks[i])
            i += 1
            expect(":")
            expect("v")
            expect(":")
            v = number_run()
            expect("x")
            expect(":")
            x = number_run()
            if v.size != nv or x.size != npos:
                raise ValueError(f"{path}: section {desc!r} t={t}: {v.size}/{x.size} values, expected {nv}/{npos}")
            sec.times.append(t)
            sec.vel.append(v)
            sec.pos.append(x)
        out.append(sec)
    return out


def _quat_angle(q1, q2):
    # Quaternion.rotationAngle (maspack/matrix/Quaternion.java:1494-1511)
    s1, u1 = q1[0], np.asarray(q1[1:4])
    s2, u2 = q2[0], np.asarray(q2[1:4])
    stmp = s1 * s2 + u1 @ u2
    utmp = np.cross(u2, u1) + s1 * u2 - s2 * u1
    ang = 2 * math.atan2(np.linalg.norm(utmp), stmp)
    return max(2 * math.pi - ang, 0.0) if ang > math.pi else ang


class _Err:
    def __init__(self, mag=0.0):
        self.err, self.mag, self.time = 0.0, mag, 0.0

    def add(self, d, m1, m2, t):
        e = float(np.linalg.norm(d))
        if e > self.err:
            self.err, self.time = e, t
        self.mag = max(self.mag, float(max(np.linalg.norm(m1), np.linalg.norm(m2))))

    def normalized(self):
        return self.err / self.mag if self.mag != 0 else self.err


def compare_sections(s1: Section, s2: Section):
    """(velocity error, position error, time of each) of one section pair."""
    if s1.description != s2.description:
        raise ValueError(f"inconsistent sections: {s1.description!r} vs {s2.description!r}")
    if s1.comps != s2.comps:
        raise ValueError(f"inconsistent components in {s1.description!r}")
    pv, av, rv = _Err(), _Err(), _Err()
    pp, ap, rp = _Err(), _Err(1.0), _Err()
    for t1, t2, v1, v2, x1, x2 in zip(s1.times, s2.times, s1.vel, s2.vel, s1.pos, s2.pos):
        if t1 != t2:
            raise ValueError(f"inconsistent times {t1} vs {t2} in {s1.description!r}")
        iv = ix = 0
        for c in s1.comps:
            if c == "P":
                pv.add(v1[iv:iv + 3] - v2[iv:iv + 3], v1[iv:iv + 3], v2[iv:iv + 3], t1)
                pp.add(x1[ix:ix + 3] - x2[ix:ix + 3], x1[ix:ix + 3], x2[ix:ix + 3], t1)
                iv += 3
                ix += 3
            elif c == "F":
                pv.add(v1[iv:iv + 3] - v2[iv:iv + 3], v1[iv:iv + 3], v2[iv:iv + 3], t1)
                av.add(v1[iv + 3:iv + 6] - v2[iv + 3:iv + 6], v1[iv + 3:iv + 6], v2[iv + 3:iv + 6], t1)
                pp.add(x1[ix:ix + 3] - x2[ix:ix + 3], x1[ix:ix + 3], x2[ix:ix + 3], t1)
                e = _quat_angle(x1[ix + 3:ix + 7], x2[ix + 3:ix + 7]) / math.pi
                if e > ap.err:
                    ap.err, ap.time = e, t1
                iv += 6
                ix += 7
            else:
                n = _sizes(c)[0]
                rv.add(v1[iv:iv + n] - v2[iv:iv + n], v1[iv:iv + n], v2[iv:iv + n], t1)
                rp.add(x1[ix:ix + n] - x2[ix:ix + n], x1[ix:ix + n], x2[ix:ix + n], t1)
                iv += n
                ix += n
    ve = max((pv, av, rv), key=lambda d: d.normalized())
    pe = max((pp, ap, rp), key=lambda d: d.normalized())
    return ve.normalized(), pe.normalized(), ve.time, pe.time


def compare_files(path1: str, path2: str, show_level: int = 0, out=sys.stdout):
    """Maximum normalised velocity and position errors over all sections
    (CompareStateFiles.compareFiles); show_level 1 prints each section's."""
    a, b = read_file(path1), read_file(path2)
    if len(a) != len(b):
        raise ValueError(f"{path1} has {len(a)} sections, {path2} {len(b)}")
    best = {"vel": (0.0, None, 0.0), "pos": (0.0, None, 0.0)}
    for s1, s2 in zip(a, b):
        ve, pe, vt, pt = compare_sections(s1, s2)
        if show_level > 0:
            print(f"{s1.description}:\nvel error={ve:.6g}\npos error={pe:.6g}", file=out)
        if ve > best["vel"][0]:
            best["vel"] = (ve, s1.description, vt)
        if pe > best["pos"][0]:
            best["pos"] = (pe, s1.description, pt)
    if show_level > -1:
        for k in ("vel", "pos"):
            e, d, t = best[k]
            print(f"max {k} error={e:.6g} at '{d}', time {t}", file=out)
    return best["vel"][0], best["pos"][0]


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    show = 0
    files = []
    for a in argv:
        if a == "-a":
            show = 1
        elif a.startswith("-"):
            print("Usage: [-a] <stateFile1> <stateFile2>")
            return 1
        else:
            files.append(a)
    if len(files) != 2:
        print("Usage: [-a] <stateFile1> <stateFile2>")
        return 1
    ve, pe = compare_files(files[0], files[1], show)
    return 0 if (ve == 0 and pe == 0) else 2


if __name__ == "__main__":
    sys.exit(main())
