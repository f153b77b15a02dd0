"""Lane-by-lane restatement, in Python, of the warp schedule that the
reinjection kernel uses for the SCEPTIC orbit-angle integral
(pot_b200/csrc/pot_inject.cu, d_integrate_for_alpha_warp; the reference's
sequential loop is pot.c:433-492).  Test infrastructure: it checks that the
schedule -- which interval each ballot picks, and the second interval a
round takes when its start was guessed -- accumulates exactly the values of
the sequential loop.  IEEE double arithmetic with the C library's exp and
sqrt, as the oracle's C code uses."""
import math

LANES = 32


def _sqrt(v):
    return math.sqrt(v) if v >= 0.0 else math.nan


def _div(a, b):
    if b == 0.0:
        return math.copysign(math.inf, a) * math.copysign(1.0, b)
    return a / b


def _y(e, chu2, s2, rol):
    y = 1.0 - (chu2 * e * math.exp(rol * (1.0 - (1.0 / e))))
    return _div(1.0, _sqrt((y / s2) - (e * e)))


def _first(mask):
    return (mask & -mask).bit_length() - 1


def warp_alpha(s, chi_b, u2, rol, mld, stats=None):
    """The warp schedule's alpha; stats (a dict) counts rounds and rounds
    that took two intervals."""
    chu2 = chi_b / u2
    s2 = s * s
    y_one = _div(s, _sqrt(1.0 - chu2 - s2))
    if s == 0.0:
        return 0.0
    alpha, xi0, y0 = 0.0, 0.0, s
    while True:
        if stats is not None:
            stats["rounds"] = stats.get("rounds", 0) + 1
        # quick round: lanes 0-7 halvings 1-8 from xi0; group g = 1..3
        # (lanes 8g..8g+7) the next interval, started at e_{g+1}
        Y, E = [0.0] * LANES, [0.0] * LANES
        for lane in range(LANES):
            grp, j = lane >> 3, lane & 7
            x_lo = xi0
            if grp:
                x_lo = 1.0
                for _ in range(grp + 1):
                    x_lo = (xi0 + x_lo) / 2.0
            ep = 1.0
            for _ in range(j + 1):
                ep = (x_lo + ep) / 2.0
            E[lane], Y[lane] = ep, _y(ep, chu2, s2, rol)
        YEK, EK, pass_all = [0.0] * LANES, [0.0] * LANES, 0
        for lane in range(LANES):
            grp, j = lane >> 3, lane & 7
            y_lo = Y[grp] if grp else y0
            YEK[lane] = y_one if j == 0 else Y[lane - 1]
            EK[lane] = 1.0 if j == 0 else E[lane - 1]
            if not (abs(YEK[lane] - Y[lane] - (Y[lane] - y_lo)) > mld):
                pass_all |= 1 << lane
        if pass_all & 0xFF:
            k = _first(pass_all & 0xFF)
            alpha += (EK[k] - xi0) * (y0 + (4.0 * Y[k]) + YEK[k]) / 6.0
            xi0, y0 = EK[k], YEK[k]
            if not (xi0 < 1.0):
                return alpha
            pass2 = (pass_all >> (8 * (k - 1))) & 0xFF if 2 <= k <= 4 else 0
            if pass2:
                if stats is not None:
                    stats["two"] = stats.get("two", 0) + 1
                k2 = 8 * (k - 1) + _first(pass2)
                alpha += (EK[k2] - xi0) * (y0 + (4.0 * Y[k2]) + YEK[k2]) / 6.0
                xi0, y0 = EK[k2], YEK[k2]
                if not (xi0 < 1.0):
                    return alpha
            continue
        # full batch: halvings 1-32 from xi0, then beyond from e_32
        top, y_top = 1.0, y_one
        while True:
            Y, E = [0.0] * LANES, [0.0] * LANES
            for lane in range(LANES):
                e = top
                for _ in range(lane + 1):
                    e = (xi0 + e) / 2.0
                E[lane], Y[lane] = e, _y(e, chu2, s2, rol)
            passed = 0
            for lane in range(LANES):
                y_hi = y_top if lane == 0 else Y[lane - 1]
                if not (abs(y_hi - Y[lane] - (Y[lane] - y0)) > mld):
                    passed |= 1 << lane
            if passed:
                k = _first(passed)
                xk = top if k == 0 else E[k - 1]
                yk = y_top if k == 0 else Y[k - 1]
                alpha += (xk - xi0) * (y0 + (4.0 * Y[k]) + yk) / 6.0
                xi0, y0 = xk, yk
                break
            if not (E[31] > xi0):
                return math.nan  # the kernel reports the halving cap here
            top, y_top = E[31], Y[31]
        if not (xi0 < 1.0):
            return alpha
