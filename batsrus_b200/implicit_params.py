"""Parameters of the implicit JFNK step (#IMPLICIT, #IMPLSTEP, #KRYLOV,
#KRYLOVSIZE, #PRECONDITIONER, #JACOBIAN; defaults of src/ModPartImplicit.f90:
52-85 and ImplParam :66-77, with the Krylov restart and preconditioner of the
implicit workload)."""
from dataclasses import dataclass


@dataclass
class ImplicitParams:
    cflImpl: float = 20.0          # CflImpl (#IMPLICIT)
    implCoeff0: float = 1.0        # ImplCoeff (#IMPLSTEP)
    useBdf2: bool = True           # UseBDF2 (#IMPLSTEP)
    nOrderImpl: int = 1            # nOrderImpl (#IMPLSCHEME)
    typeFluxImpl: str = "default"  # TypeFluxImpl (#IMPLSCHEME)
    jacobianEps: float = 1e-12     # JacobianEps (#JACOBIAN)
    nKrylovVector: int = 30        # GMRES(30) (#KRYLOVSIZE)
    maxMatvec: int = 100           # MaxMatvec (#KRYLOV)
    errorMax: float = 1e-3         # relative tolerance (#KRYLOV)
    typePrecond: str = "BILU"      # BILU | NONE | LEARNED (#PRECONDITIONER)
    precondPrecision: str = "fp64"  # BILU factors: fp64 (the reference's) | fp32 | bf16 (FP32 factorisation)


def apply_implicit_commands(commands, p):
    for name, v in commands:
        if name == "#IMPLICIT":
            if bool(v[1]) or bool(v[2]):
                p.cflImpl = float(v[3])
        elif name in ("#IMPLSTEP", "#IMPLICITSTEP"):
            p.implCoeff0 = float(v[0])
            p.useBdf2 = bool(v[1])
        elif name in ("#IMPLSCHEME", "#IMPLICITSCHEME"):
            p.nOrderImpl = int(v[0])
            p.typeFluxImpl = str(v[1])
        elif name == "#JACOBIAN":
            p.jacobianEps = float(v[1])
        elif name == "#KRYLOV":
            p.errorMax = float(v[2])
            p.maxMatvec = int(v[3])
        elif name == "#KRYLOVSIZE":
            p.nKrylovVector = int(v[0])
        elif name == "#PRECONDITIONER":
            p.typePrecond = str(v[1]).upper()
    return p
