/*
 * lbm_oracle_st.c -- CPU restatement of the reference's D3Q7 solute
 * (passive scalar) update, TEST INFRASTRUCTURE (rules as in lbm_oracle.c).
 *
 * Restates Single_Phase_3D/Solute_Transport_MPI_Software_Spars_6V.cpp
 * ("ST7") for a fully periodic domain: `init` (ST7:1249-1327) sets
 * g_k = C/6 (1 + 3 e_k.u) for the six axis velocities e2 (ST7:130) with the
 * velocity array as it is before the velocity file is read (main calls init
 * at ST7:472 and Backup_input_v at :473), i.e. zero: g_k = C/6; each step is
 * `collision` (ST7:1345-1617: BGK g -> g - (g - C/6 (1 + 3 e.u))/tau_s with
 * the file's velocity, push streaming with halfway bounce-back LR,
 * ST7:1475-1528) followed by `comput_macro_variables` (ST7:1619-1633:
 * C = sum_k g_k, k = 1..6).
 *
 * Pinned bit for bit against the reference program itself, run as two ranks
 * of its x-slab decomposition under the multi-process MPI stand-in
 * (oracle/mpishim, oracle/_ref/ref_st7_slab; fixture tests/golden/st7_slab.npz),
 * and by the physics (mass conservation, pure diffusion with variance 2 D t
 * where D = (tau_s - 1/2)/3, advection of the centroid at u).
 *
 * Layout: ids 1..count in SP3 compaction order, g AoS [(count+1)*7] (slot 0
 * unused, as in the reference), u AoS [(count+1)*3], C [(count+1)].
 * The neighbour table is the D3Q19 nei_loc of lbm_oracle.c (its first seven
 * directions are e2).
 */
#include <stdint.h>
#include <string.h>

static const int E7[7][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
static const int LR7[7] = {0, 2, 1, 4, 3, 6, 5};

/* tau_s = niu_s / (c_s^2 dt) + 0.5 (ST7:1262) */
double orc_st7_tau(double diffusivity) {
  const double c_s2 = 1.0 * 1.0 / 3, dt = 1.0;
  return diffusivity / (c_s2 * dt) + 0.5;
}

void orc_st7_init(int count, const double* c0, double* g, double* C) {
  memset(g, 0, sizeof(double) * 7);
  C[0] = 0;
  for (int i = 1; i <= count; i++) {
    C[i] = c0[i];
    g[(long)i * 7 + 0] = 0.0;
    for (int lm = 1; lm < 7; lm++) {
      const double eu = 0.0;  /* the velocity array before the velocity file is read */
      g[(long)i * 7 + lm] = 1.0 / 6.0 * C[i] * (1 + 3 * eu);
    }
  }
}

/* nei is the D3Q19 push table [(count+1)*19]; directions 1..6 are e2. */
void orc_st7_step(int count, const int32_t* nei, const double* u, double tau_s, double* g, double* G, double* C) {
  for (int ci = 1; ci <= count; ci++) {
    double gr[7];
    for (int mi = 1; mi < 7; mi++) {
      const double eu = E7[mi][0] * u[(long)ci * 3 + 0] + E7[mi][1] * u[(long)ci * 3 + 1] + E7[mi][2] * u[(long)ci * 3 + 2];
      const double f = g[(long)ci * 7 + mi];
      gr[mi] = f - (f - 1.0 / 6.0 * C[ci] * (1 + 3 * eu)) / tau_s;
    }
    for (int mi = 1; mi < 7; mi++) {
      const int32_t d = nei[(long)ci * 19 + mi];
      if (d > 0)
        G[(long)d * 7 + mi] = gr[mi];
      else
        G[(long)ci * 7 + LR7[mi]] = gr[mi];
    }
  }
  for (int i = 1; i <= count; i++) {
    double c = 0;
    for (int k = 1; k < 7; k++) {
      g[(long)i * 7 + k] = G[(long)i * 7 + k];
      c += g[(long)i * 7 + k];
    }
    C[i] = c;
  }
}
