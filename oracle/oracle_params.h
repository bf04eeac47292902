/*
 * Test infrastructure only (the oracle): the physics parameters passed to both
 * CPU oracles (oracle/astaroth_oracle.c and the reference model built by
 * oracle/ref_driver.cc).  The names are those of the reference's run_const
 * params (acc-runtime/samples/mhd_modular/mhdsolver.ac:230-251).
 */
#pragma once

typedef struct {
    double ds[3];
    double nu_visc;
    double eta;
    double cs_sound;
    double gamma;
    double cp_sound;
    double lnrho0;
    double lnT0;
    double mu0;
    double zeta;
    double K_heatcond;
    int upwind; /* 1: the LUPWD terms (restatement only; the reference model
                   takes LUPWD at compile time, libastaroth_ref_upwd.so) */
    /* helical forcing in substep 2 (restatement: when forcing != 0; the
     * reference model built with LFORCING=1 always applies it) */
    int forcing;
    double f_magnitude, f_phase, f_kaver;
    double f_k[3], f_re[3], f_im[3];
} OracleParams;
