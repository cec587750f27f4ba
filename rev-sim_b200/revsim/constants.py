"""Physical constants and default force-field parameters of the 3-site water model.

Values follow greener-group/rev-sim ``water/water.jl``:

* masses and temperature: ``water.jl:43-46``
* reaction-field constant k_rf = (1/rc^3)(78.3-1)/(2*78.3+1): ``water.jl:41``
* cutoffs 1.0 nm (interaction) / 1.2 nm (neighbour list), rebuild every 20 steps,
  snapshot every 1000 steps: ``water.jl:37-40,42``
* test parameters (sigma, eps, alpha, beta, A, B, C, q_O, k_b, r0, k_a, theta0):
  ``water.jl:1562-1582``
* enthalpy-of-vaporisation loss: mean gas-phase energy 3.69, RT 2.45 and the target
  44.12 + 2.8 kJ/mol: ``water.jl:738-755``

Units are nm, ps, u (g/mol), kJ/mol, K and elementary charges.  The Coulomb constant
and Boltzmann constant come from the CODATA 2018 SI definitions (the reference reads
them from Molly/Unitful); k_B in kJ mol^-1 K^-1 equals u nm^2 ps^-2 K^-1.
"""

import math

O_MASS = 15.99943
H_MASS = 1.007947
TEMP = 295.15
KB = 0.00831446261815324
COULOMB_CONST = 138.93545764438196

DIST_CUTOFF = 1.0
DIST_NEIGHBORS = 1.2
N_STEPS_NF = 20
N_STEPS_LOG = 1000
CRF_CONST = (1.0 / DIST_CUTOFF**3) * ((78.3 - 1) / (2 * 78.3 + 1))

ENTH_U_GAS, ENTH_RT, ENTH_TARGET = 3.69, 2.45, 44.12 + 2.8

# Pair forms in the order of water.jl:121-150 (generate_inter).
INTER_TYPES = {"lj": 0, "dexp": 1, "buck": 2, "ljsc": 3, "buff": 4}
N_FORM_PARAMS = {"lj": 2, "dexp": 4, "buck": 3, "ljsc": 4, "buff": 4}

SIGMA = 0.315
EPSILON = 0.636
DEXP_ALPHA, DEXP_BETA = 16.766, 4.427
BUCK_A, BUCK_B, BUCK_C = 133996.0, 27.6, 0.0168849
LJSC_ALPHA, LJSC_LAMBDA = 0.2, 0.1
BUFF_DELTA, BUFF_GAMMA = 0.07, 0.12
O_CHARGE = -0.834
KB_BOND, R0_BOND = 462750.4, 0.09572
KA_ANGLE, THETA0_ANGLE = 836.8, 1.82421813418


def default_params(inter_type="lj", beta=None):
    """Parameter vector in the reference layout (water.jl:1572-1582):
    pair-form parameters, then q_O, k_b, r0, k_a, theta0."""
    tail = [O_CHARGE, KB_BOND, R0_BOND, KA_ANGLE, THETA0_ANGLE]
    if inter_type == "lj":
        head = [SIGMA, EPSILON]
    elif inter_type == "dexp":
        head = [SIGMA, EPSILON, DEXP_ALPHA, DEXP_BETA if beta is None else beta]
    elif inter_type == "buck":
        head = [BUCK_A, BUCK_B, BUCK_C]
    elif inter_type == "ljsc":
        head = [SIGMA, EPSILON, LJSC_ALPHA, LJSC_LAMBDA]
    elif inter_type == "buff":
        head = [SIGMA, EPSILON, BUFF_DELTA, BUFF_GAMMA]
    else:
        raise ValueError("inter_type not recognised")
    return head + tail


def n_params(inter_type):
    return N_FORM_PARAMS[inter_type] + 5


def langevin_coeffs(gamma, dt):
    """c = exp(-gamma dt), s = sqrt(1 - c^2) (water.jl:1019-1020)."""
    c = math.exp(-gamma * dt)
    return c, math.sqrt(1 - c * c)


# ------------------------------------------------------------------ gas in water
# diffusion.jl: 885 waters and 10 O2 in a 3.0 nm box (:30-34, :47), O2 bond
# k = 1640.4 kcal mol^-1 A^-2 and r0 = 0.12074 nm (:46, :1113-1116), gas sites of mass m_O
# and no charge; default sigma_gas / eps_gas and the per-form parameters (:1621-1639).
GAS_N_WATER, GAS_N_GAS, GAS_BOX = 885, 10, 3.0
GAS_KB_BOND, GAS_R0_BOND = 1640.4 * 4.184 * 100, 0.12074
GAS_SIGMA, GAS_EPSILON = 0.3297, 0.438
GAS_BUCK = (BUCK_A, BUCK_B, BUCK_C)
GAS_LOSS_TYPES = {"diff": 1, "ev": 4, "diff_ev": 5}


def gas_default_params(inter_type="lj"):
    """Parameter vector of diffusion.jl:1629-1639: the water and gas pair-form parameters,
    the form's own globals, then q_O."""
    if inter_type == "lj":
        head = [SIGMA, EPSILON, GAS_SIGMA, GAS_EPSILON]
    elif inter_type == "dexp":
        head = [SIGMA, EPSILON, GAS_SIGMA, GAS_EPSILON, DEXP_ALPHA, DEXP_BETA]
    elif inter_type == "buck":
        head = [BUCK_A, BUCK_B, BUCK_C, *GAS_BUCK]
    elif inter_type == "ljsc":
        head = [SIGMA, EPSILON, GAS_SIGMA, GAS_EPSILON, LJSC_ALPHA, LJSC_LAMBDA]
    elif inter_type == "buff":
        head = [SIGMA, EPSILON, GAS_SIGMA, GAS_EPSILON, BUFF_DELTA, BUFF_GAMMA]
    else:
        raise ValueError("inter_type not recognised")
    return head + [O_CHARGE]


def gas_n_params(inter_type):
    return 5 if inter_type == "lj" else 7
