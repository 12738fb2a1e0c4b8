"""Synthetic cross-section generator for the Full-Penn inelastic and Kieft-Bosch
elastic scatter models, in the layout of Nebula's material files.

Nebula's material file (read by ``io/hdf5_file.cpp`` and consumed by
``full_penn::create`` ``physics/full_penn.h:294-406`` and
``kieft_elastic::create`` ``physics/kieft/elastic.h:120-166``) holds, per
material:

====================== ============================== ======== ==================
dataset                axes (dimension scales)        unit     consumer
====================== ============================== ======== ==================
/elastic/imfp          K (log, eV)                    nm^-1    elastic.h:129-140
/elastic/costheta_icdf K (log, eV) x P (lin)          --       elastic.h:144-157
/full_penn/imfp        K (log, eV)                    nm^-1    full_penn.h:306-317
/full_penn/omega_icdf  K (log, eV) x P (lin)          eV       full_penn.h:321-344
/full_penn/q_icdf      K (log, eV) x w/K (lin) x P    nm^-1    full_penn.h:348-369
/ionization/binding_icdf K (log) x w/K (log) x P      eV       full_penn.h:374-402
====================== ============================== ======== ==================

plus the properties ``fermi``, ``barrier``, ``band_gap``, ``phonon_loss`` (eV)
and ``effective_A`` (mass per atom, g).

The physics used to fill the tables (all in float64):

* elastic: screened Rutherford, dsigma/dOmega = Z(Z+1) (e^2/(4 pi eps0) / (2E))^2
  / (1 - cos t + 2 eta)^2 with Moliere's screening parameter
  eta = (1/4) (hbar/(p a_TF))^2 (1.13 + 3.76 (alpha Z / beta)^2),
  a_TF = 0.88534 a0 Z^(-1/3).  The angular ICDF is analytic:
  mu = (1 - cos t)/2 = eta P / (1 + eta - P).
* inelastic: a single-pole Drude-Lindhard energy-loss function
  Im[-1/eps(q, w)] = wp^2 g w / ((w^2 - wq^2)^2 + (g w)^2), wq = wp + q^2
  (q in units of hbar q / sqrt(2m), i.e. eV^1/2), and the plane-wave DIIMFP
  d(1/lambda)/dw = 1/(pi a0 K) int_{q-}^{q+} dq/q Im[-1/eps(q, w)],
  q+- = sqrt(K) +- sqrt(K - w), with w limited to K - E_F.
* no inner shells: the binding table is all zeros, which ``full_penn::create``
  maps to -1 (Fermi-sea excitation only).

``build_raw_material(spec, inelastic="kieft")`` writes the tables of the
Kieft-Bosch inelastic model instead of Full Penn's
(``kieft_inelastic::create`` ``physics/kieft/inelastic.h:215-331``):

========================== ========================== ======== ==================
/inelastic_kieft/imfp      K (log, eV)                nm^-1    inelastic.h:226-238
/inelastic_kieft/w0_icdf   K (log, eV) x P (lin)      eV       inelastic.h:240-261
/ionization/binding_icdf   K (log, eV) x P (lin)      eV       inelastic.h:262-327
/ionization/outer_shells   shell index                eV       inelastic.h:270-282
========================== ========================== ======== ==================

* the inverse mean free path is the same Drude-Lindhard one;
* the zero-momentum loss w' follows the optical-data model (Ashley 1988):
  d(1/lambda)/dw' = 1/(pi a0 K) Im[-1/eps(0, w')] L(w'/K), with
  L(x) = (1-x) ln(4/x) - 7x/4 + x^(3/2) - 33x^2/32 clipped at 0;
* inner shells (binding >= 50 eV) take a Bethe-like share of the events,
  f(K) = c ln(K/B) / (K/B) above B, placed at the top of the probability
  axis; the rest of the axis is 0 (no inner shell);
* outer shells: the valence binding energies of the material's elements.

Everything here is seeded-free and deterministic: the same call gives the
same bytes.
"""
from __future__ import annotations

import dataclasses
import numpy as np

A0_NM = 0.052917721          # Bohr radius (nm)
HBARC_EVNM = 197.3269804     # hbar c (eV nm)
MC2_EV = 510998.95           # electron rest energy (eV)
ALPHA = 1.0 / 137.035999     # fine-structure constant
E2_EVNM = 1.439964548        # e^2 / (4 pi eps0) (eV nm)
Q_UNIT_NM_SQRT_EV = 0.19519  # hbar/sqrt(2 m) in nm eV^1/2 (full_penn.h:359)
AMU_G = 1.66053907e-24       # atomic mass unit (g)


@dataclasses.dataclass
class MaterialSpec:
    """Physical constants of one synthetic material."""
    name: str
    Z: float                 # (average) atomic number for screened Rutherford
    atom_density: float      # atoms per nm^3
    plasmon: float           # Drude pole energy wp (eV)
    damping: float           # Drude damping g (eV)
    fermi: float             # Fermi energy (eV)
    work_function: float     # work function (eV)
    band_gap: float          # band gap (eV); -1 means metal
    phonon_loss: float       # acoustic phonon loss (eV)
    effective_A: float       # atomic mass (u)
    e_min: float = 1.0       # table energy range (eV)
    e_max: float = 10e3
    n_energy: int = 64
    n_prob: int = 64
    n_wk: int = 64           # w/K axis of the q ICDF

    @property
    def barrier(self) -> float:
        return self.fermi + self.work_function


def silicon(e_max: float = 10e3) -> MaterialSpec:
    """Si-like material: Z=14, wp=16.6 eV, g=4 eV, E_F=7.8, W=4.8, gap 1.1."""
    return MaterialSpec("silicon", Z=14.0, atom_density=49.94, plasmon=16.6,
                        damping=4.0, fermi=7.8, work_function=4.8, band_gap=1.1,
                        phonon_loss=0.05, effective_A=28.0855, e_max=e_max)


# Kieft-Bosch model: (binding eV, share scale c) of the inner shells and the
# valence (outer-shell) binding energies, per material name (Si: 2p, 2s, 1s;
# 3p, 3s.  PMMA: C 1s, O 1s; C 2p, O 2p, C 2s).
INNER_SHELLS = {"silicon": [(99.42, 0.06), (149.7, 0.02), (1839.0, 0.01)],
                "pmma": [(284.2, 0.05), (543.1, 0.02)]}
OUTER_SHELLS = {"silicon": [8.15, 13.46], "pmma": [11.26, 13.62, 16.59]}


def pmma(e_max: float = 10e3) -> MaterialSpec:
    """PMMA-like material: average Z=6.5, wp=19 eV, W=4.5 eV.

    Not fixed by the workload definition and chosen here: damping 4 eV,
    E_F 7.0 eV, band gap 5.6 eV, phonon loss 0.05 eV, A = 100.12/15 u and
    1.07e23 atoms/cm^3 (1.19 g/cm^3 C5H8O2).
    """
    return MaterialSpec("pmma", Z=6.5, atom_density=107.4, plasmon=19.0,
                        damping=4.0, fermi=7.0, work_function=4.5, band_gap=5.6,
                        phonon_loss=0.05, effective_A=100.12 / 15.0, e_max=e_max)


# ----------------------------------------------------------------------------
# elastic
def moliere_eta(E, Z):
    E = np.asarray(E, dtype=np.float64)
    pc = np.sqrt(E * E + 2.0 * E * MC2_EV)
    gam = 1.0 + E / MC2_EV
    beta = np.sqrt(1.0 - 1.0 / gam ** 2)
    a_tf = 0.88534 * A0_NM * Z ** (-1.0 / 3.0)
    return 0.25 * (HBARC_EVNM / pc / a_tf) ** 2 * (1.13 + 3.76 * (ALPHA * Z / beta) ** 2)


def elastic_imfp(E, spec: MaterialSpec):
    """Inverse elastic mean free path (nm^-1), screened Rutherford."""
    E = np.asarray(E, dtype=np.float64)
    eta = moliere_eta(E, spec.Z)
    sigma = (E2_EVNM / (2.0 * E)) ** 2 * spec.Z * (spec.Z + 1.0) * np.pi / (eta * (1.0 + eta))
    return spec.atom_density * sigma


def elastic_costheta_icdf(E, P, spec: MaterialSpec):
    eta = moliere_eta(E, spec.Z)[:, None]
    P = np.asarray(P)[None, :]
    mu = eta * P / (1.0 + eta - P)
    return np.clip(1.0 - 2.0 * mu, -1.0, 1.0)


# ----------------------------------------------------------------------------
# inelastic
def drude_lindhard_elf(q, w, spec: MaterialSpec):
    wq = spec.plasmon + q * q
    g = spec.damping
    return spec.plasmon ** 2 * g * w / ((w * w - wq * wq) ** 2 + (g * w) ** 2)


def _q_grid(K, w, n):
    """Log-spaced q grid between q- and q+ (eV^1/2), shape (..., n)."""
    sk = np.sqrt(K)
    skw = np.sqrt(np.maximum(K - w, 0.0))
    qm = np.maximum(sk - skw, 1e-12)
    qp = sk + skw
    t = np.linspace(0.0, 1.0, n)
    return np.exp(np.log(qm)[..., None] + (np.log(qp) - np.log(qm))[..., None] * t)


def _q_integral(K, w, spec, n=256):
    """int_{q-}^{q+} dq/q ELF(q, w), integrated in log q."""
    q = _q_grid(K, w, n)
    f = drude_lindhard_elf(q, np.asarray(w)[..., None], spec)
    lq = np.log(q)
    return np.trapezoid(f, lq, axis=-1)


def inelastic_tables(spec: MaterialSpec, energies, probs, n_w=1024):
    """Return (imfp[K], omega_icdf[K, P]) for the Drude-Lindhard DIIMFP."""
    imfp = np.empty(len(energies))
    omega = np.empty((len(energies), len(probs)))
    for i, K in enumerate(energies):
        w_hi = K - spec.fermi
        if w_hi <= 2e-3:
            imfp[i] = 1e-30
            omega[i, :] = max(w_hi, 1e-3)
            continue
        w = np.exp(np.linspace(np.log(1e-3), np.log(w_hi), n_w))
        dens = _q_integral(np.full_like(w, K), w, spec) / (np.pi * A0_NM * K)
        # cumulative in w (trapezoid)
        cdf = np.concatenate([[0.0], np.cumsum(0.5 * (dens[1:] + dens[:-1]) * np.diff(w))])
        total = cdf[-1]
        imfp[i] = max(total, 1e-30)
        cdf = cdf / total if total > 0 else np.linspace(0, 1, len(w))
        # make strictly increasing for interpolation
        cdf = np.maximum.accumulate(cdf + np.arange(len(cdf)) * 1e-15)
        cdf /= cdf[-1]
        omega[i, :] = np.interp(probs, cdf, w)
    return imfp, omega


def q_icdf_table(spec: MaterialSpec, energies, wk, probs, n_q=256):
    """q ICDF (eV^1/2) over (K, w/K, P)."""
    out = np.empty((len(energies), len(wk), len(probs)))
    for i, K in enumerate(energies):
        w = np.clip(np.asarray(wk) * K, 1e-6 * K, K)
        q = _q_grid(np.full_like(w, K), w, n_q)                 # (nw, nq)
        f = drude_lindhard_elf(q, w[:, None], spec) / q          # density in q
        cdf = np.concatenate([np.zeros((len(w), 1)),
                              np.cumsum(0.5 * (f[:, 1:] + f[:, :-1]) * np.diff(q, axis=1), axis=1)],
                             axis=1)
        for j in range(len(w)):
            c = cdf[j]
            if not np.isfinite(c[-1]) or c[-1] <= 0:
                out[i, j, :] = q[j, 0]
                continue
            c = c / c[-1]
            c = np.maximum.accumulate(c + np.arange(len(c)) * 1e-15)
            c /= c[-1]
            out[i, j, :] = np.interp(probs, c, q[j])
    return out


def ashley_L(x):
    x = np.asarray(x, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        v = (1 - x) * np.log(4 / x) - 1.75 * x + x ** 1.5 - 33.0 / 32.0 * x * x
    return np.where(np.isfinite(v) & (v > 0), v, 0.0)


def kieft_w0_icdf(spec: MaterialSpec, energies, probs, n_w=1024):
    """ICDF of the zero-momentum loss w' (eV) over (K, P), optical-data model."""
    out = np.empty((len(energies), len(probs)))
    for i, K in enumerate(energies):
        w_hi = K - spec.fermi
        if w_hi <= 2e-3:
            out[i, :] = max(w_hi, 1e-3)
            continue
        w = np.exp(np.linspace(np.log(1e-3), np.log(w_hi), n_w))
        dens = drude_lindhard_elf(0.0, w, spec) * ashley_L(w / K)
        cdf = np.concatenate([[0.0], np.cumsum(0.5 * (dens[1:] + dens[:-1]) * np.diff(w))])
        if not np.isfinite(cdf[-1]) or cdf[-1] <= 0:
            out[i, :] = w[0]
            continue
        cdf = cdf / cdf[-1]
        cdf = np.maximum.accumulate(cdf + np.arange(len(cdf)) * 1e-15)
        cdf /= cdf[-1]
        out[i, :] = np.interp(probs, cdf, w)
    return out


def kieft_binding_icdf(spec: MaterialSpec, energies, probs):
    """Binding energy (eV) over (K, P): inner shells at the top of the P axis
    with Bethe-like shares, 0 (no inner shell) elsewhere."""
    out = np.zeros((len(energies), len(probs)))
    for i, K in enumerate(energies):
        top = 1.0
        for B, c in INNER_SHELLS.get(spec.name, []):
            if K <= B:
                continue
            u = K / B
            share = c * np.log(u) / u * np.e          # peaks at c for K = e B
            lo = top - share
            out[i, (probs >= lo) & (probs < top)] = B
            if top >= 1.0:
                out[i, probs >= 1.0] = B
            top = lo
    return out


# ----------------------------------------------------------------------------
def build_raw_material(spec: MaterialSpec, inelastic: str = "full_penn") -> dict:
    """Raw material content (datasets with dimension scales, properties).

    The result has the structure of a Nebula material file: it is what
    ``nebula_b200.synth.nmat.write`` serialises and what both the C++ loader
    and the HDF5 stand-in used to compile the reference read.
    """
    K = np.geomspace(spec.e_min, spec.e_max, spec.n_energy)
    P = np.linspace(0.0, 1.0, spec.n_prob)
    WK = np.linspace(0.0, 1.0, spec.n_wk)

    el_imfp = elastic_imfp(K, spec)
    el_icdf = elastic_costheta_icdf(K, P, spec)
    props = {
        "fermi": (spec.fermi, "eV"),
        "barrier": (spec.barrier, "eV"),
        "band_gap": (spec.band_gap, "eV"),
        "phonon_loss": (spec.phonon_loss, "eV"),
        "effective_A": (spec.effective_A * AMU_G, "g"),
        "work_function": (spec.work_function, "eV"),
    }
    if inelastic == "kieft":
        in_imfp, _ = inelastic_tables(spec, K, P)
        datasets = {
            "/elastic/imfp": dict(unit="nm^-1", data=el_imfp, scales=[("eV", K)]),
            "/elastic/costheta_icdf": dict(unit="", data=el_icdf, scales=[("eV", K), ("", P)]),
            "/inelastic_kieft/imfp": dict(unit="nm^-1", data=in_imfp, scales=[("eV", K)]),
            "/inelastic_kieft/w0_icdf": dict(unit="eV", data=kieft_w0_icdf(spec, K, P), scales=[("eV", K), ("", P)]),
            "/ionization/binding_icdf": dict(unit="eV", data=kieft_binding_icdf(spec, K, P),
                                             scales=[("eV", K), ("", P)]),
            "/ionization/outer_shells": dict(unit="eV", data=np.asarray(OUTER_SHELLS[spec.name], np.float64),
                                             scales=[None]),
        }
        return dict(name=spec.name, datasets=datasets, properties=props)
    if inelastic != "full_penn":
        raise ValueError("inelastic model must be 'full_penn' or 'kieft'")
    in_imfp, omega = inelastic_tables(spec, K, P)
    q = q_icdf_table(spec, K, WK, P)

    Kb = np.geomspace(spec.e_min, spec.e_max, 2)
    Wb = np.geomspace(1e-3, 1.0, 2)
    Pb = np.linspace(0.0, 1.0, 2)

    datasets = {
        "/elastic/imfp": dict(unit="nm^-1", data=el_imfp, scales=[("eV", K)]),
        "/elastic/costheta_icdf": dict(unit="", data=el_icdf, scales=[("eV", K), ("", P)]),
        "/full_penn/imfp": dict(unit="nm^-1", data=in_imfp, scales=[("eV", K)]),
        "/full_penn/omega_icdf": dict(unit="eV", data=omega, scales=[("eV", K), ("", P)]),
        "/full_penn/q_icdf": dict(unit="nm^-1", data=q / Q_UNIT_NM_SQRT_EV,
                                  scales=[("eV", K), ("", WK), ("", P)]),
        "/ionization/binding_icdf": dict(unit="eV", data=np.zeros((2, 2, 2)),
                                         scales=[("eV", Kb), ("", Wb), ("", Pb)]),
    }
    return dict(name=spec.name, datasets=datasets, properties=props)
