"""Algorithmic bytes of one step.

The roofline numerator (``minimal_member_bytes``) is the compulsory DRAM traffic of the MINIMAL phase decomposition of
the benchmark member (air stack L = 3 + ocean stack L = 2, three FCT tracers each, nfast = 20): a phase boundary only
where a grid-wide dependency forces one (the step's free surface; per stage the cells-and-vertices pass, the edges
pass, two passes per barotropic sub-step, the flux limiter and the update; five FCT cell passes), each array charged
once per phase at its stored width. At level 6 that is 870.7 MB for the air stack and 804.5 MB for the ocean stack
per step in the FP64 form, 738 MB and 687 MB in the mixed form; other levels scale with the edge count.

``layers_step_bytes`` / ``transport_bytes`` count the same way over THIS core's own decomposition, which has more
phases (the packed edge record between E and S, phase C apart from D, the FCT's edge-flux passes), so they charge
more bytes (1,954 MB for the level-6 member): a figure for comparing the core's phases, not the roofline's.

Each phase (one grid-wide pass between two grid-wide dependencies) is charged every array it reads or writes once, at
its stored width, as if nothing stayed on chip between phases: index tables int32 (signs and slots int8), geometry and
state FP64. A gather that touches a neighbour's value is not charged again (the array is charged once per phase).
achieved = minimal bytes / measured time, against the measured HBM copy bandwidth. At level 6 a member's working set
(tens of MB) fits in the 126 MB L2, so the DRAM bytes ncu reports fall below these figures: the phases run from L2.
"""

import math

I4, I1, F8 = 4, 1, 8

LEVEL6_EDGES = 122880
MINIMAL_MEMBER_BYTES_L6 = {'double': 870.7e6 + 804.5e6, 'mixed': 738e6 + 687e6}


def minimal_member_bytes(E, form='double'):
    """Compulsory bytes of one member step (air 3 + ocean 2 layers, 3 tracers each, nfast 20) on a grid of E edges."""
    return MINIMAL_MEMBER_BYTES_L6[form] * E / LEVEL6_EDGES


def layers_step_bytes(N, E, NV, nE2, L, nfast, nu4=True, vmix=False, Fm=True):
    """Bytes of one time-split RK3 step of L layers (the launch sequence in csrc/layers.cu)."""
    cell_tab = 6 * N * I4 + 6 * N * I1        # cellEdge + cellSign
    asc_tab = 6 * N * I4                      # cellEdgeAsc
    e2c = 2 * E * I4                          # eI, eJ
    e2v = 2 * E * I4                          # ev1, ev2
    v_tab = 3 * NV * I4 + 3 * NV * I1         # vEdge + vEdgeSign
    vc_tab = 3 * NV * I4 + 3 * NV * I1        # vCell + vSlot
    LN, LE, LV = L * N * F8, L * E * F8, L * NV * F8
    b = 0
    # init: eta0 (cells) and ubar0 (edges)
    b += LN + N * F8 + N * F8 + e2c + LE + E * F8
    if nu4:
        # twice: D and zeta (cells + vertices), then the edge Laplacian
        lap_cv = LE + cell_tab + E * F8 + N * F8 + v_tab + E * F8 + NV * F8 + LN + LV
        lap_e = LN + LV + e2c + e2v + 2 * E * F8 + LE
        b += 2 * (lap_cv + lap_e)
    cs = (1 / 3, 1 / 2, 1.0)
    for s, c in enumerate(cs):
        n = max(1, math.ceil(c * nfast))
        # A: B (cells) and q (vertices)
        b += LN + LE + N * F8 + cell_tab + 2 * E * F8 + N * F8 + N * F8 + LN + N * F8
        b += vc_tab + 6 * N * F8 + v_tab + NV * F8 + NV * F8 + LV
        # E: h_e, packed (h_e, u, q_e), ubar and acc reset
        b += LN + LV + LE + e2c + e2v + E * F8 + LE + 3 * LE + 2 * E * F8
        # S: slow tendencies
        b += 3 * LE + nE2 * F8 + (E + 1) * I4 + nE2 * I4 + LE + LE + LN + e2c + E * F8 + (LE if nu4 else 0) + LE + 3 * E * F8
        # fast loop: eta (cells) then ubar (edges), n times
        bt_eta = 2 * E * F8 + cell_tab + E * F8 + N * F8 + N * F8 + 2 * N * F8
        bt_u = 2 * N * F8 + N * F8 + E * F8 + e2c + E * F8 + 2 * E * F8 + 2 * E * F8
        b += n * (bt_eta + bt_u)
        # C: layer fluxes and the floor limiter's scale
        b += asc_tab + e2c + 3 * E * F8 + LN + LE + LN + N * F8 + LE + LN
        # D: h_n (cells), Fm and u_n (edges)
        b += cell_tab + E * F8 + LE + LN + e2c + LN + N * F8 + LN
        b += 2 * E * F8 + LE + LE + LE + (LE if (Fm and s == 2) else 0)
    if vmix and L > 1:
        b += LN + e2c + 2 * LE + E * F8
    return b


def transport_bytes(N, E, L, T, order=3):
    """Bytes of mass_after plus one step_many of T tracers (csrc/transport.cu)."""
    R = T * L
    LN, LE, RN, RE = L * N * F8, L * E * F8, R * N * F8, R * E * F8
    asc, e2c = 6 * N * I4, 2 * E * I4
    d2 = 8 * E * I4 + 8 * E * F8
    b = LN + LE + asc + e2c + LN                                     # mass_after
    b += RN + 2 * LN + LE + asc + e2c + (d2 if order == 3 else 0) + RN + RN + (RN if order == 3 else 0)   # P1
    if order == 3:
        b += RN + RN + LN + LE + asc + e2c + d2 + RN                 # P2
        b += 3 * RN + LN + LE + 6 * N * I4 + asc + e2c + d2 + RE + 2 * RN   # P3
        b += RN + LN + RE + 2 * RN + asc + e2c + RN                  # P4
    else:
        b += RN + RN
    return b


def grid_sizes(g):
    return int(g.N), int(g.E), int(g.NV), int(g.eoeStart[-1])
