"""Scenes whose optics depend on the wavelength, with closed forms integrated
over the sun's spectrum. No reference test solves with a multi-node sun and
wavelength-dependent materials (the reference pins only a monochromatic sun
through a spectral extinction, src/test_ssol_solver1.c:491-528), so each scene
here carries its own expectation: the mean of a per-wavelength closed form
over the density of the wavelength sampler, the sun spectrum read as a
piecewise-linear function (src/ssol_ranst_sun_wl.c:84-105)."""
import math

import numpy as np

import material_scenes as M
import pyssol as P
import ref_scenes as R

SUN_WL = [0.4, 0.6, 0.8, 1.0]
SUN_I = [0.5, 1.0, 0.8, 0.3]
SPAN = [0.4, 1.0]


def spectral_mean(f):
    """Mean of the vectorised f(wavelengths) over the sun spectrum."""
    wl = np.linspace(SUN_WL[0], SUN_WL[-1], 400001)
    p = np.interp(wl, SUN_WL, SUN_I)
    return float(np.trapezoid(f(wl) * p, wl) / np.trapezoid(p, wl))


def refl_of(wl):
    """Heliostat reflectivity; linear in the wavelength, so a tabulation at
    the sun's nodes interpolates it exactly."""
    return 0.3 + 0.5 * wl


def k_of(wl):
    return np.interp(wl, SPAN, [0.05, 0.01])


def n_of(wl):
    return np.interp(wl, SPAN, [1.65, 1.4])


def alpha_of(wl):
    return np.interp(wl, SPAN, [40.0, 5.0])


def sun(s, direction):
    s.set_sun("directional", direction, R.DNI, spectrum=s.spectrum(SUN_WL, SUN_I))


def solver1_spectral(lib):
    """The scene of src/test_ssol_solver1.c:402-485 (primary sampled only,
    heliostat replaced, atmosphere) with a reflectivity refl_of(wl) and an
    extinction k_of(wl): the target receives
    4 DNI cos45 E_wl[refl(wl) exp(-k(wl) 4 sqrt2)]."""
    s, h = R.solver1_base(lib)
    lib.call("ssol_instance_sample", h["target"], 0)
    lib.call("ssol_instance_sample", h["secondary"], 0)
    lib.call("ssol_scene_detach_instance", s.scn, h["heliostat"])
    m2 = s.mirror(lambda wl, frag: float(refl_of(wl)), 0.0)
    s.instance(s.object([(h["square"], m2, m2)]), receiver=P.SSOL_FRONT)
    sun(s, (1, 0, -1))
    s.atmosphere(s.spectrum(SPAN, [0.05, 0.01]))
    d = 4 * math.sqrt(2)
    expected = 4 * R.DNI * R.COS45 * spectral_mean(lambda wl: refl_of(wl) * np.exp(-k_of(wl) * d))
    return s, {"receiver": h["target"], "expected": expected}


def glass_spectral(lib):
    """The glass plate of material_scenes.glass_slab with n(wl) from 1.65 to
    1.4 under the vertical sun: DNI A E_wl[(1 - R) / (1 + R)],
    R = ((n - 1) / (n + 1))^2."""
    s = P.Scene(lib)
    air = s.medium(0.0, 1.0)
    glass = s.medium(0.0, s.spectrum(SPAN, [1.65, 1.4]))
    enter, leave = s.dielectric(air, glass), s.dielectric(glass, air)
    v = s.virtual()
    s.instance(s.object([(s.rectangle(5, 5), v, v)]), P.transform_from(None, (0, 0, 2.0)))
    s.instance(s.object([(s.rectangle(5, 5), enter, leave)]),
               P.transform_from(None, (0, 0, 1.0)), sample=0)
    s.instance(s.object([(s.rectangle(5, 5), enter, leave)]),
               P.transform_from(P.rotation_pitch_pi(), (0, 0, 0.9)), sample=0)
    absorber = s.matte(0.0)
    rcv = s.instance(s.object([(s.rectangle(10, 10), absorber, absorber)]),
                     receiver=P.SSOL_FRONT, sample=0)
    sun(s, (0, 0, -1))

    def passed(wl):
        r = M.fresnel_normal(1.0, n_of(wl))
        return (1 - r) / (1 + r)
    return s, {"receiver": rcv, "expected": M.DNI * M.AREA * spectral_mean(passed)}


def thin_slab_spectral(lib, thickness=0.005):
    """The thin-dielectric window with n(wl) and absorption(wl) spectra:
    DNI A E_wl[(1 - R)^2 tau / (1 - R^2 tau^2)], tau = exp(-alpha thickness)."""
    s = P.Scene(lib)
    air = s.medium(0.0, 1.0)
    slab = s.medium(s.spectrum(SPAN, [40.0, 5.0]), s.spectrum(SPAN, [1.65, 1.4]))
    win = s.thin_dielectric(air, slab, thickness)
    v = s.virtual()
    s.instance(s.object([(s.rectangle(5, 5), v, v)]), P.transform_from(None, (0, 0, 2.0)))
    s.instance(s.object([(s.rectangle(5, 5), win, win)]), P.transform_from(None, (0, 0, 1.0)),
               sample=0)
    absorber = s.matte(0.0)
    rcv = s.instance(s.object([(s.rectangle(10, 10), absorber, absorber)]),
                     receiver=P.SSOL_FRONT, sample=0)
    sun(s, (0, 0, -1))

    def passed(wl):
        r = M.fresnel_normal(1.0, n_of(wl))
        tau = np.exp(-alpha_of(wl) * thickness)
        return (1 - r) ** 2 * tau / (1 - r * r * tau * tau)
    return s, {"receiver": rcv, "expected": M.DNI * M.AREA * spectral_mean(passed)}


BUILDERS = {"solver1": solver1_spectral, "glass": glass_spectral,
            "thin_slab": thin_slab_spectral}
