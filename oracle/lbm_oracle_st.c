/* D3Q7 solute restatement (test infrastructure); see lbm_oracle.c for conventions. */
