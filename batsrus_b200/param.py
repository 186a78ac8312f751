"""PARAM.in reader for the commands this hot path honours.

The reference reads PARAM.in with share/Library ModReadParam (absent from the
tree) and dispatches the commands in src/ModSetParameters.f90
(``set_parameters``).  A command is a line starting with ``#NAME``; its
parameters follow one per line (value first, anything after the value is a
comment) until a blank line.  ``#RUN`` ends a session, ``#END`` the file.
Lines that do not start with ``#`` outside a command are comments.

Supported here (others are kept in ``Session.commands`` and ignored):

* ``#SCHEME nOrder TypeFlux [TypeLimiter [LimiterBeta]]``
  (src/ModSetParameters.f90:1745-1779; PARAM.XML:7158-7238)
* ``#TIMESTEPPING`` / ``#RUNGEKUTTA`` / ``#RK nStage CflExpl`` (:628-633)
* ``#FIXEDTIMESTEP UseDtFixed DtFixedDim`` (:649-650, Cfl=1 :4317-4321)
* ``#GAMMA``, ``#GRID``, ``#OUTERBOUNDARY``, ``#CHECKGRIDSIZE``, ``#STOP``,
  ``#DIVB`` (UseDivbSource), ``#UPDATE``, ``#CONSERVEFLUX``, ``#TIMEACCURATE``
* initial states: ``#SHOCKTUBE``, ``#SHOCKPOSITION``, ``#UNIFORMSTATE``,
  ``#WAVE`` (src/ModSetInitialCondition.f90:74-150)
* implicit solvers: ``#IMPLICIT``, ``#IMPLSTEP``, ``#KRYLOV``, ``#KRYLOVSIZE``,
  ``#PRECONDITIONER``, ``#NEWTON``, ``#JACOBIAN``, ``#SEMIIMPLICIT``,
  ``#SEMIKRYLOV``, ``#SEMIPRECOND`` (src/ModPartImplicit.f90:116-248,
  src/ModSemiImplicit.f90:51-108)
"""
from dataclasses import dataclass, field


def _value(tok):
    t = tok.strip()
    if t in ("T", ".true.", "TRUE", "true"):
        return True
    if t in ("F", ".false.", "FALSE", "false"):
        return False
    try:
        return int(t)
    except ValueError:
        pass
    try:
        return float(t.replace("d", "e").replace("D", "e"))
    except ValueError:
        return t


def read_param(text):
    """Return a list of sessions; each session is a list of (command, values)."""
    sessions, cur = [], []
    lines = text.splitlines()
    n = 0
    while n < len(lines):
        line = lines[n]
        n += 1
        s = line.strip()
        if not s.startswith("#"):
            continue
        name = s.split()[0].upper()
        if name == "#END":
            break
        if name == "#RUN":
            sessions.append(cur)
            cur = []
            continue
        vals = []
        while n < len(lines) and lines[n].strip() != "":
            tok = lines[n].split("\t")[0].split()
            # the value is the first whitespace-separated token unless the line
            # holds a multi-word string (e.g. "1d mhd idl_ascii")
            raw = lines[n].split("\t")[0].strip()
            vals.append(_value(tok[0]) if len(tok) == 1 else raw)
            n += 1
        cur.append((name, vals))
    if cur:
        sessions.append(cur)
    return sessions


@dataclass
class Scheme:
    """Numerical scheme of one session (defaults: src/ModSetParameters.f90:
    set_defaults :3141-3155, src/ModFaceValue.f90:51-52, src/ModMain.f90:36)."""
    nOrder: int = 2
    nStage: int = 2
    typeFlux: str = "Rusanov"
    typeLimiter: str = "minmod"
    limiterBeta: float = 1.0
    cfl: float = 0.8
    gamma: float = 5.0 / 3.0
    useDivbSource: bool = True
    useDtFixed: bool = False
    dtFixed: float = 0.0
    useHalfStep: bool = True
    isTimeAccurate: bool = True
    precision: str = "fp64"  # 'fp64' | 'fp32'
    useNonConservative: bool = False  # #NONCONSERVATIVE (oracle only; the GPU path solves for energy)
    # floors (#MINIMUMDENSITY / #MINIMUMPRESSURE / #MINIMUMTEMPERATURE,
    # normalized units), active where > 0 (RhoMinDim_I = pMinDim_I =
    # TMinDim_I = -1 by default, src/ModPhysics.f90:170-172); massIon in amu
    # #RESOLUTIONCHANGE (src/ModFaceValue.f90:44-76): TVD faces at
    # resolution changes (the reference's default), the softer limiter near
    # them when limiterBeta > betaLimiterResChange
    useTvdResChange: bool = True
    betaLimiterResChange: float = 2.0
    nFaceLimiterResChange: int = 2
    rhoMin: float = -1.0
    pMin: float = -1.0
    tMin: float = -1.0
    massIon: float = 1.0


@dataclass
class Session:
    scheme: Scheme
    commands: list = field(default_factory=list)
    tSimulationMax: float = -1.0
    maxIteration: int = -1


def apply_commands(commands, scheme, nDim=3):
    """Apply one session's commands on top of ``scheme`` (in place)."""
    info = {}
    for name, v in commands:
        if name == "#SCHEME":
            scheme.nOrder = int(v[0])
            scheme.nStage = scheme.nOrder
            scheme.useHalfStep = scheme.nStage <= 2
            scheme.typeFlux = str(v[1])
            scheme.limiterBeta = 1.0
            if scheme.nOrder > 1 and scheme.typeFlux.upper() != "SIMPLE":
                scheme.typeLimiter = str(v[2])
                if scheme.typeLimiter not in ("minmod", "no"):
                    scheme.limiterBeta = float(v[3])
            else:
                scheme.typeLimiter = "no"
        elif name in ("#TIMESTEPPING", "#RUNGEKUTTA", "#RK"):
            scheme.nStage = int(v[0])
            scheme.cfl = float(v[1])
            scheme.useHalfStep = name == "#TIMESTEPPING" and scheme.nStage <= 2
        elif name == "#FIXEDTIMESTEP":
            scheme.useDtFixed = bool(v[0])
            if scheme.useDtFixed:
                scheme.dtFixed = float(v[1])
        elif name == "#GAMMA":
            scheme.gamma = float(v[0])
        elif name == "#DIVB":
            scheme.useDivbSource = bool(v[0])
        elif name == "#RESOLUTIONCHANGE":  # src/ModFaceValue.f90:168-177
            if bool(v[0]):
                raise ValueError("#RESOLUTIONCHANGE: UseAccurateResChange is not on the GPU path")
            scheme.useTvdResChange = bool(v[1])
            scheme.betaLimiterResChange = float(v[2])
            scheme.nFaceLimiterResChange = int(v[3])
        elif name == "#TVDRESCHANGE":  # :182-184
            scheme.useTvdResChange = bool(v[0])
        elif name == "#MINIMUMDENSITY":  # src/ModSetParameters.f90:706-709
            scheme.rhoMin = float(v[0])
        elif name == "#MINIMUMPRESSURE":  # :711-714
            scheme.pMin = float(v[0])
        elif name == "#MINIMUMTEMPERATURE":  # :717-720
            scheme.tMin = float(v[0])
        elif name == "#TIMEACCURATE":
            scheme.isTimeAccurate = bool(v[0])
        elif name == "#STOP":
            info["maxIteration"] = int(v[0])
            info["tSimulationMax"] = float(v[1])
        else:
            info.setdefault(name, []).append(v)
    if scheme.useDtFixed:
        scheme.cfl = 1.0  # UseDtFixed only works with Cfl = 1 (:4317-4321)
    return info
