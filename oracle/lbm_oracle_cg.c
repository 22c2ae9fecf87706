/* Colour-gradient two-phase restatement (test infrastructure); see lbm_oracle.c for conventions. */
