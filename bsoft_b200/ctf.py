"""CTF parameters as the reference defines them (host side).

``CTFparam`` (bsoft/include/ctf.h:28-460) stores the CTF as aberration
weights ``abw[{n,m}]``:

* abw[0,0]  = -amplitude phase shift, where the shift is asin(amp_contrast)
  when a STAR file gives ``ctf.amp_contrast`` (rwmgSTAR.cpp:481-484);
* abw[2,0]  = t2 * defocus_average,  t2 = -pi * lambda     (ctf.h:133-134, 76-78);
* abw[2,+2] = t2 * dev * cos(2 ang), abw[2,-2] = t2 * dev * sin(2 ang) (ctf.h:137-141);
* abw[4,0]  = t1 * Cs, t1 = pi/2 * lambda^3               (ctf.h:143-144);
* abw[1,+-1] = 2 pi * beam tilt                           (ctf.h:128-131).

Even aberration phase (ctf.h:321-334), with s2 = |s|^2 and a = atan2(sy, sx):
  chi = abw00 + s2*(abw2m2*sin 2a + abw20 + abw22*cos 2a) + s2^2*abw40.
Odd aberration phase (ctf.h:335-348): psi = |s|*(abw1m1*sin a + abw11*cos a).
Electron wavelength (ctf.h:309-317).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

PLANCK = 6.626070e-34
EMASS = 9.109384e-31
ECHARGE = 1.602177e-19
LIGHTSPEED = 299792458.0


def electron_wavelength(volt: float) -> float:
    """Relativistic electron wavelength in angstrom for an accelerating
    voltage in volts (ctf.h:309-317)."""
    if volt <= 0:
        return 0.0
    return PLANCK * 1e10 / math.sqrt(
        2.0 * EMASS * ECHARGE * volt * (1.0 + ECHARGE * volt / (2.0 * EMASS * LIGHTSPEED * LIGHTSPEED)))


@dataclass
class CTFParams:
    volt: float = 300000.0          # V
    cs: float = 2.7e7               # angstrom
    amp_shift: float = 0.0          # radians (asin of amplitude contrast)
    defocus: float = 20000.0        # angstrom, positive = underfocus
    def_dev: float = 0.0            # angstrom
    ast_angle: float = 0.0          # radians
    beam_tilt_x: float = 0.0        # radians
    beam_tilt_y: float = 0.0

    @staticmethod
    def from_amp_contrast(volt, cs, amp_contrast, defocus, def_dev=0.0, ast_angle=0.0):
        return CTFParams(volt=volt, cs=cs, amp_shift=math.asin(amp_contrast),
                         defocus=defocus, def_dev=def_dev, ast_angle=ast_angle)

    def coefficients(self) -> np.ndarray:
        """[abw00, abw20, abw22, abw2m2, abw40, abw11, abw1m1] in radians per
        the appropriate power of 1/angstrom."""
        wl = electron_wavelength(self.volt)
        t1 = math.pi / 2 * wl * wl * wl
        t2 = -math.pi * wl
        dev = abs(self.def_dev)
        return np.array([
            -self.amp_shift,
            t2 * self.defocus,
            t2 * dev * math.cos(2 * self.ast_angle),
            t2 * dev * math.sin(2 * self.ast_angle),
            t1 * self.cs,
            2 * math.pi * self.beam_tilt_x,
            2 * math.pi * self.beam_tilt_y,
        ], dtype=np.float64)


def ctf_chi(coef: np.ndarray, s2: np.ndarray, ang: np.ndarray) -> np.ndarray:
    abw00, abw20, abw22, abw2m2, abw40 = coef[:5]
    return abw00 + s2 * (abw2m2 * np.sin(2 * ang) + abw20 + abw22 * np.cos(2 * ang)) + s2 * s2 * abw40


def ctf_image(coef: np.ndarray, n: int, pixel: float) -> np.ndarray:
    """sin(chi) on the unshifted n x n FFT grid (frequency index wrapped at
    (n-1)/2 as Bimage does)."""
    f = np.arange(n, dtype=np.float64)
    f[f > (n - 1) // 2] -= n
    f /= (n * pixel)
    sy, sx = np.meshgrid(f, f, indexing="ij")
    s2 = sx * sx + sy * sy
    return np.sin(ctf_chi(coef, s2, np.arctan2(sy, sx)))
