"""Closed-form scenes for the rows that no reference test pins: dielectric
interfaces, thin dielectric slabs and the Russian roulette. Vertical sun,
10x10 squares; expectations follow from Fresnel at normal incidence."""
import pyssol as P

DNI = 1000.0
AREA = 100.0


def fresnel_normal(n1, n2):
    return ((n1 - n2) / (n1 + n2)) ** 2


def glass_slab(lib, n_glass=1.5, thickness=0.1):
    """A glass plate (two parallel 10x10 faces) above a 20x20 receiver.

    Top face (front up): outside air / inside glass; its back side (seen from
    inside the glass) has the media swapped. Bottom face flipped (front down)
    with the same rule, so that a ray always meets the material whose
    outside medium is the one it travels in. Expected receiver incoming flux
    at normal incidence, no absorption: DNI A (1 - R) / (1 + R)."""
    s = P.Scene(lib)
    sq = s.rectangle(5, 5)
    air = s.medium(0.0, 1.0)
    glass = s.medium(0.0, n_glass)
    enter = s.dielectric(air, glass)
    leave = s.dielectric(glass, air)
    # A sampled point on a dielectric starts inside its "inside" medium
    # (src/ssol_solver.c:307-316), so the sun is sampled on a virtual plane
    # above the glass instead.
    v = s.virtual()
    s.instance(s.object([(s.rectangle(5, 5), v, v)]), P.transform_from(None, (0, 0, 2.0)))
    top = s.instance(s.object([(sq, enter, leave)]), P.transform_from(None, (0, 0, 1.0)),
                     sample=0)
    bottom_obj = s.object([(s.rectangle(5, 5), enter, leave)])
    bot = s.instance(bottom_obj, P.transform_from(P.rotation_pitch_pi(), (0, 0, 1.0 - thickness)),
                     sample=0)
    rcv_shape = s.rectangle(10, 10)
    absorber = s.matte(0.0)
    rcv = s.instance(s.object([(rcv_shape, absorber, absorber)]), receiver=P.SSOL_FRONT,
                     sample=0)
    s.set_sun("directional", (0, 0, -1), DNI)
    R = fresnel_normal(1.0, n_glass)
    return s, {"receiver": rcv, "top": top, "bottom": bot,
               "expected": DNI * AREA * (1 - R) / (1 + R)}


def thin_slab(lib, n_glass=1.5, absorption=20.0, thickness=0.005):
    """A thin dielectric 10x10 window above a 20x20 absorbing receiver.
    Expected incoming flux at normal incidence:
    DNI A (1 - R)^2 tau / (1 - R^2 tau^2), tau = exp(-absorption thickness)."""
    import math
    s = P.Scene(lib)
    sq = s.rectangle(5, 5)
    air = s.medium(0.0, 1.0)
    slab = s.medium(absorption, n_glass)
    win = s.thin_dielectric(air, slab, thickness)
    v = s.virtual()
    s.instance(s.object([(s.rectangle(5, 5), v, v)]), P.transform_from(None, (0, 0, 2.0)))
    s.instance(s.object([(sq, win, win)]), P.transform_from(None, (0, 0, 1.0)), sample=0)
    absorber = s.matte(0.0)
    rcv = s.instance(s.object([(s.rectangle(10, 10), absorber, absorber)]),
                     receiver=P.SSOL_FRONT, sample=0)
    s.set_sun("directional", (0, 0, -1), DNI)
    R = fresnel_normal(1.0, n_glass)
    tau = math.exp(-absorption * thickness)
    return s, {"receiver": rcv, "expected": DNI * AREA * (1 - R) ** 2 * tau / (1 - R * R * tau * tau)}


def light_trap(lib, gap=1.0, tan_theta=0.09):
    """Two perfect 10x10 mirrors `gap` apart under a directional sun tilted
    by theta from the vertical. The upper one reflects on its lower face and
    is virtual on its upper face, so the sun reaches the lower mirror and
    light bounces between them, drifting gap tan(theta) sideways per
    segment until it leaves through a side: up to 10 / (gap tan theta)
    bounces, so the Russian roulette (first at depth 65, then every 16) ends
    about half the paths and doubles the weight of each survivor. Every
    sampled watt is eventually missing, so whatever the roulette does,
    E[missing] = DNI x 100 cos(theta) and E[cos_factor] = cos(theta).
    The depth stays below 4 x 16 + 3 x 16 + 1, so no path carries a weight
    above 8 and the sample variance is honest."""
    import math
    s = P.Scene(lib)
    m = s.mirror(1.0, 0.0)
    v = s.virtual()
    low = s.instance(s.object([(s.rectangle(5, 5), m, m)]))
    # rotated by pi: the front (mirror) faces down, the back (virtual) up,
    # so the shadow ray of the sun sees the virtual side
    up_obj = s.object([(s.rectangle(5, 5), m, v)])
    s.instance(up_obj, P.transform_from(P.rotation_pitch_pi(), (0, 0, gap)), sample=0)
    c = 1 / math.sqrt(1 + tan_theta ** 2)
    s.set_sun("directional", (tan_theta * c, 0.0, -c), DNI)
    return s, {"low": low, "cos": c, "expected_missing": DNI * AREA * c}
