"""IMEX Runge-Kutta methods for the segregated Runge-Kutta step of the collocated scheme
(Solver.srk_init / tc_srk_init): the method families of collocated_SRK/imex.h:10-41 with
their published double Butcher tables.

Each table has (S + 1) x S entries, row-major: rows 0..S-1 are the stage coefficients
a_ij, the last row the weights b_j.  `kind` is the formulation the reference's step uses
for the method (ARS: explicit first stage; CK: Kennedy-Carpenter type with the extra
nu1tilde / d_j terms).  Coefficients written as ratios of integers are evaluated as
float(p) / float(q), as a C++ compiler evaluates `p./q.`.

    ARS_121, ARS_232, ARS_343   Ascher, Ruuth, Spiteri, Appl. Numer. Math. 25 (1997)
    MARS_343                    Boscarino, Russo, SIAM J. Sci. Comput. 31 (2009)
    ARK3, ARK4                  Kennedy, Carpenter, Appl. Numer. Math. 44 (2003):
                                ARK3(2)4L[2]SA, ARK4(3)6L[2]SA
    MARK3                       Boscarino, Russo: MARK3(2)4L[2]SA
    BHR_553                     Boscarino, J. Comput. Phys. 228 (2009)
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

A, ARS, CK = 0, 1, 2  # TC_IMEX_A, TC_IMEX_ARS, TC_IMEX_CK

# middle root of 6x^3 - 18x^2 + 9x - 1 = 0 (the L-stable SDIRK diagonal)
GAMMA3 = 0.435866521508458999416019451193556842529


def _q(p: int, q: int) -> float:
    return float(p) / float(q)


@dataclass
class Method:
    name: str
    kind: int
    S: int
    E: list = field(default_factory=list)  # explicit table, (S+1) x S
    I: list = field(default_factory=list)  # implicit table, (S+1) x S
    alpha_tau_max: tuple = (2.0, 2.0)  # stability limit for StabType 0 and 1

    def check(self):
        n = self.S * (self.S + 1)
        if len(self.E) != n or len(self.I) != n:
            raise ValueError(f"{self.name}: tables must have (S+1) x S = {n} entries")
        return self

    def alpha_tau(self, stab_type: int) -> float:
        """The value the reference's driver uses: half the stability limit."""
        return 0.5 * self.alpha_tau_max[stab_type]


def calc_d(S: int, A_: list) -> list:
    """Coefficients d_j of the CK formulation (collocated_SRK/imex.cpp:37-46)."""
    a_ss = A_[S * S - 1]
    d = [1.0] + [0.0] * (S - 1)
    for j in range(1, S):
        for k in range(j):
            d[j] -= A_[j * S + k] * d[k] / a_ss
    return d


def order_sums(S: int, A_: list) -> tuple:
    """Residuals of the order conditions up to 3 for one table (b = last row):
    sum b - 1, 2 b.c - 1, 3 b.c^2 - 1, 6 b.A.c - 1 with c_i = sum_j a_ij
    (the checks of collocated_SRK/imex.cpp:7-33)."""
    b = A_[S * S:]
    a = [A_[i * S:(i + 1) * S] for i in range(S)]
    s1 = sum(b) - 1.0
    s2 = sum(2.0 * b[j] * a[j][k] for j in range(S) for k in range(S)) - 1.0
    s31 = sum(3.0 * b[j] * a[j][k] * a[j][l] for j in range(S) for k in range(S) for l in range(S)) - 1.0
    s32 = sum(6.0 * b[j] * a[j][k] * a[k][l] for j in range(S) for k in range(S) for l in range(S)) - 1.0
    return s1, s2, s31, s32


def ARS_121() -> Method:
    return Method("ARS_121", ARS, 2, E=[0., 0., 1., 0., 0., 1.], I=[0., 0., 0., 1., 0., 1.]).check()


def ARS_232() -> Method:
    g = 1. - 0.5 * math.sqrt(2.)
    dl = -2. * math.sqrt(2.) / 3.
    E = [0., 0., 0.,
         g, 0., 0.,
         dl, 1. - dl, 0.,
         0., 1. - g, g]
    I = [0., 0., 0.,
         0., g, 0.,
         0., 1. - g, g,
         0., 1. - g, g]
    return Method("ARS_232", ARS, 3, E=E, I=I).check()


def ARS_343() -> Method:
    g = GAMMA3
    b1 = -1.5 * g * g + 4 * g - 0.25
    b2 = 1.5 * g * g - 5. * g + 1.25
    I = [0., 0., 0., 0.,
         0., g, 0., 0.,
         0., (1. - g) / 2., g, 0.,
         0., b1, b2, g,
         0., b1, b2, g]
    a42 = 0.5529291479
    a43 = a42
    a31 = (1. - 4.5 * g + 1.5 * g * g) * a42 + (2.75 - 10.5 * g + 3.75 * g * g) * a43 - 3.5 + 13. * g - 4.5 * g * g
    a32 = -(1. - 4.5 * g + 1.5 * g * g) * a42 - (2.75 - 10.5 * g + 3.75 * g * g) * a43 + 4. - 12.5 * g + 4.5 * g * g
    E = [0., 0., 0., 0.,
         g, 0., 0., 0.,
         a31, a32, 0., 0.,
         1. - a42 - a43, a42, a43, 0.,
         0., b1, b2, g]
    return Method("ARS_343", ARS, 4, E=E, I=I).check()


def MARS_343() -> Method:
    g = GAMMA3
    b2 = 1.20849664917601
    I = [0., 0., 0., 0.,
         0., g, 0., 0.,
         0., 0.28206673924577, g, 0.,
         0., b2, 1. - g - b2, g,
         0., b2, 1. - g - b2, g]
    E = [0., 0., 0., 0.,
         g, 0., 0., 0.,
         0.535396540307354, 0.182536720446875, 0., 0.,
         0.63041255815287, -0.83193390106308, 1.20152134291021, 0.,
         0., b2, 1. - g - b2, g]
    return Method("MARS_343", ARS, 4, E=E, I=I).check()


def ARK3() -> Method:
    g = GAMMA3
    b1 = _q(1471266399579, 7840856788654)
    b2 = _q(-4482444167858, 7529755066697)
    b3 = 1. - g - b1 - b2
    I = [0., 0., 0., 0.,
         g, g, 0., 0.,
         _q(2746238789719, 10658868560708), _q(-640167445237, 6845629431997), g, 0.,
         b1, b2, b3, g,
         b1, b2, b3, g]
    E = [0., 0., 0., 0.,
         2 * g, 0., 0., 0.,
         _q(5535828885825, 10492691773637), _q(788022342437, 10882634858940), 0., 0.,
         _q(6485989280629, 16251701735622), _q(-4246266847089, 9704473918619), _q(10755448449292, 10357097424841), 0.,
         b1, b2, b3, g]
    return Method("ARK3", CK, 4, E=E, I=I).check()


def ARK4() -> Method:
    b = [_q(82889, 524892), 0., _q(15625, 83664), _q(69875, 102672), _q(-2260, 8211), 0.25]
    I = [0., 0., 0., 0., 0., 0.,
         0.25, 0.25, 0., 0., 0., 0.,
         _q(8611, 62500), _q(-1743, 31250), 0.25, 0., 0., 0.,
         _q(5012029, 34652500), _q(-654441, 2922500), _q(174375, 388108), 0.25, 0., 0.,
         _q(15267082809, 155376265600), _q(-71443401, 120774400), _q(730878875, 902184768), _q(2285395, 8070912), 0.25, 0.,
         *b,
         *b]
    E = [0., 0., 0., 0., 0., 0.,
         0.5, 0., 0., 0., 0., 0.,
         _q(13861, 62500), _q(6889, 62500), 0., 0., 0., 0.,
         _q(-116923316275, 2393684061468), _q(-2731218467317, 15368042101831), _q(9408046702089, 11113171139209), 0., 0., 0.,
         _q(-451086348788, 2902428689909), _q(-2682348792572, 7519795681897), _q(12662868775082, 11960479115383),
         _q(3355817975965, 11060851509271), 0., 0.,
         _q(647845179188, 3216320057751), _q(73281519250, 8382639484533), _q(552539513391, 3454668386233),
         _q(3354512671639, 8306763924573), _q(4040, 17871), 0.,
         *b]
    return Method("ARK4", CK, 6, E=E, I=I).check()


def MARK3() -> Method:
    g = GAMMA3
    b1 = 0.60424832458800
    I = [0., 0., 0., 0.,
         g, g, 0., 0.,
         -4.30002662176923, 2.26541338346372, g, 0.,
         b1, 0., 1. - g - b1, g,
         b1, 0., 1. - g - b1, g]
    E = [0., 0., 0., 0.,
         2 * g, 0., 0., 0.,
         -3.06478674186224, 1.46604002506519, 0., 0.,
         0.21444560762133, 0.71075364965269, 0.07480074272597, 0.,
         b1, 0., 1. - g - b1, g]
    return Method("MARK3", CK, 4, E=E, I=I).check()


def BHR_553() -> Method:
    S = 5
    I = [0.0] * 30
    E = [0.0] * 30
    g = _q(424782, 974569)
    I[5] = I[6] = g
    I[10] = g
    I[11] = _q(-31733082319927313, 455705377221960889379854647102)
    I[12] = g
    I[15] = _q(-3012378541084922027361996761794919360516301377809610,
               45123394056585269977907753045030512597955897345819349)
    I[16] = _q(-62865589297807153294268, 102559673441610672305587327019095047)
    I[17] = _q(418769796920855299603146267001414900945214277000, 212454360385257708555954598099874818603217167139)
    I[18] = g
    I[20] = _q(487698502336740678603511, 1181159636928185920260208)
    I[22] = _q(302987763081184622639300143137943089, 1535359944203293318639180129368156500)
    I[23] = _q(-105235928335100616072938218863, 2282554452064661756575727198000)
    I[24] = g
    E[5] = 2. * g
    E[10] = g
    E[11] = g
    E[15] = _q(-475883375220285986033264, 594112726933437845704163)
    E[17] = _q(1866233449822026827708736, 594112726933437845704163)
    E[20] = _q(62828845818073169585635881686091391737610308247, 176112910684412105319781630311686343715753056000)
    E[21] = -I[22]
    E[22] = _q(262315887293043739337088563996093207, 297427554730376353252081786906492000)
    E[23] = _q(-987618231894176581438124717087, 23877337660202969319526901856000)
    for i in range(5):
        E[25 + i] = I[25 + i] = I[20 + i]
    return Method("BHR_553", CK, S, E=E, I=I).check()


METHODS = {f.__name__: f for f in (ARS_121, ARS_232, ARS_343, MARS_343, ARK3, ARK4, MARK3, BHR_553)}
