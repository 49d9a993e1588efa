/*
 * CPU oracle for the learned preconditioner: an FP64 restatement of the message-passing
 * network, its loss and its backward pass.
 *
 * TEST INFRASTRUCTURE ONLY. The network has no counterpart in the reference
 * (FreddyJuka/mpi-cst-fem-solver); this file is the independent CPU statement of the
 * network that the GPU kernels implement, used by tests/ to check the GPU forward pass and
 * the GPU gradients. The GPU library never links or calls it.
 *
 * Network (node graph = the stiffness pattern's node blocks, self excluded; F = 64):
 *   X_n   = [r/s (2), d/d_mean (2), xy/coord_scale (2), material (2)]      inputs, 8
 *   H0    = relu(W_in X + b_in)
 *   for l = 1..3:  A_l = mean over neighbours m of H_{l-1,m}
 *                  U_l = W_l [H_{l-1}; A_l] + b_l,  G_l = relu(U_l),  H_l = H_{l-1} + G_l
 *   Y     = W_out H3 + b_out                                               outputs, 2
 *   z     = D^-1 (r + s Y)             (s = RMS of r: z is homogeneous of degree 1 in r)
 * Loss per sample (r, e = A^-1 r): L = 1 - (z'r)^2 / ((z'Az)(e'r)), the squared sine of the
 * angle between z and e in the energy norm (z'Ae = z'r): 0 when z is parallel to the error.
 *
 * Parameter vector (P, 25474 values): W_in[64][8], b_in[64], (W_l[64][128], b_l[64]) x 3,
 * W_out[2][64], b_out[2]; every W row-major [out][in].
 *
 * With q = 1 the forward pass rounds what the GPU stores in BF16 (inputs, H, A) to BF16 and
 * the biases to FP32, so that GPU and oracle see the same numbers at every stored point; the
 * backward pass treats those roundings as identities (as the GPU does).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define MP_F 64
#define MP_IN 8
#define MP_L 3
#define MP_OUT 2

enum {
  OFF_WIN = 0,
  OFF_BIN = OFF_WIN + MP_F * MP_IN,
  OFF_L0 = OFF_BIN + MP_F,
  L_STRIDE = MP_F * 2 * MP_F + MP_F,
  OFF_WOUT = OFF_L0 + MP_L * L_STRIDE,
  OFF_BOUT = OFF_WOUT + MP_OUT * MP_F,
  MP_NPARAM = OFF_BOUT + MP_OUT
};

long mp_param_count(void) { return MP_NPARAM; }

/* round to nearest even at FP32, then at BF16 (what __float2bfloat16_rn of an FP32 value gives) */
static double rb(double v) {
  float f = (float)v;
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) {
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
  }
  u &= 0xffff0000u;
  memcpy(&f, &u, 4);
  return (double)f;
}
static double rf(double v) { return (double)(float)v; }

double mp_round_bf16(double v) { return rb(v); }

/* Inputs of every node (see above); m0/m1 the node's two material values. */
void mp_features(int N, const double* r, const double* invd, const double* xy, const double* mat,
                 double s, double d_mean, double coord_scale, double* X) {
  for (int n = 0; n < N; ++n) {
    double* x = X + (long)n * MP_IN;
    x[0] = r[2 * n] / s;
    x[1] = r[2 * n + 1] / s;
    x[2] = (1.0 / invd[2 * n]) / d_mean;
    x[3] = (1.0 / invd[2 * n + 1]) / d_mean;
    x[4] = xy[2 * n] / coord_scale;
    x[5] = xy[2 * n + 1] / coord_scale;
    x[6] = mat[2 * n];
    x[7] = mat[2 * n + 1];
  }
}

/* H: (MP_L + 1) * N * F, G and A: MP_L * N * F, Y: N * 2. nbr/node_ptr: the node-block pattern
 * (self included; skipped here). */
void mp_forward(int N, const int* node_ptr, const int* nbr, const double* X_in, const double* P, int q,
                double* H, double* G, double* A, double* Y) {
  const long NF = (long)N * MP_F;
  for (int n = 0; n < N; ++n) {
    for (int o = 0; o < MP_F; ++o) {
      double u = q ? rf(P[OFF_BIN + o]) : P[OFF_BIN + o];
      for (int k = 0; k < MP_IN; ++k) {
        const double xv = q ? rb(X_in[(long)n * MP_IN + k]) : X_in[(long)n * MP_IN + k];
        u += P[OFF_WIN + o * MP_IN + k] * xv;
      }
      const double h = u > 0.0 ? u : 0.0;
      H[(long)n * MP_F + o] = q ? rb(h) : h;
    }
  }
  for (int l = 0; l < MP_L; ++l) {
    const double* Hp = H + l * NF;
    double* Hn = H + (l + 1) * NF;
    double* Al = A + l * NF;
    double* Gl = G + l * NF;
    const double* W = P + OFF_L0 + l * L_STRIDE;
    const double* b = W + MP_F * 2 * MP_F;
    for (int n = 0; n < N; ++n) {
      int deg = 0;
      double acc[MP_F];
      for (int o = 0; o < MP_F; ++o) acc[o] = 0.0;
      for (int k = node_ptr[n]; k < node_ptr[n + 1]; ++k) {
        const int m = nbr[k];
        if (m == n) continue;
        ++deg;
        for (int o = 0; o < MP_F; ++o) acc[o] += Hp[(long)m * MP_F + o];
      }
      for (int o = 0; o < MP_F; ++o) {
        const double a = deg ? acc[o] / deg : 0.0;
        Al[(long)n * MP_F + o] = q ? rb(a) : a;
      }
    }
    for (int n = 0; n < N; ++n) {
      for (int o = 0; o < MP_F; ++o) {
        double u = q ? rf(b[o]) : b[o];
        const double* w = W + o * 2 * MP_F;
        for (int k = 0; k < MP_F; ++k) u += w[k] * Hp[(long)n * MP_F + k];
        for (int k = 0; k < MP_F; ++k) u += w[MP_F + k] * Al[(long)n * MP_F + k];
        const double g = u > 0.0 ? u : 0.0;
        Gl[(long)n * MP_F + o] = g;
        const double h = Hp[(long)n * MP_F + o] + g;
        Hn[(long)n * MP_F + o] = q ? rb(h) : h;
      }
    }
  }
  const double* H3 = H + MP_L * NF;
  for (int n = 0; n < N; ++n)
    for (int c = 0; c < MP_OUT; ++c) {
      double y = q ? rf(P[OFF_BOUT + c]) : P[OFF_BOUT + c];
      for (int k = 0; k < MP_F; ++k) y += P[OFF_WOUT + c * MP_F + k] * H3[(long)n * MP_F + k];
      Y[(long)n * MP_OUT + c] = y;
    }
}

/* z = D^-1 (r + s Y) */
void mp_apply(int N, const double* r, const double* invd, double s, const double* Y, double* z) {
  for (long i = 0; i < 2L * N; ++i) z[i] = invd[i] * (r[i] + s * Y[i]);
}

/* Loss of the learned multigrid cycle's output for one sample (r, e) and dL/dY: the network reads
 * r2 (the residual left after the cycle's fixed part x_fix, features and s from r2) and its
 * output is the post-smoothing step, z = x_fix + winvd (r2 + s Y), winvd = omega D^-1. The loss is
 * the same energy-norm angle as mp_loss, of z against e, on the sample's r. Returns L. */
double mp_loss_cycle(int N, const int* rp, const int* cols, const double* vals, const double* r, const double* e,
                     const double* xfix, const double* r2, const double* winvd, double s, const double* Y,
                     double* dY) {
  const long n = 2L * N;
  double c = 0.0, zaz = 0.0, er = 0.0;
  for (long i = 0; i < n; ++i) {
    const double zi = xfix[i] + winvd[i] * (r2[i] + s * Y[i]);
    c += zi * r[i];
    er += e[i] * r[i];
    double az = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = cols[k];
      az += vals[k] * (xfix[j] + winvd[j] * (r2[j] + s * Y[j]));
    }
    zaz += zi * az;
  }
  const double L = 1.0 - c * c / (zaz * er);
  if (dY) {
    const double f1 = -2.0 * c / (zaz * er), f2 = 2.0 * c * c / (zaz * zaz * er);
    for (long i = 0; i < n; ++i) {
      double az = 0.0;
      for (int k = rp[i]; k < rp[i + 1]; ++k) {
        const int j = cols[k];
        az += vals[k] * (xfix[j] + winvd[j] * (r2[j] + s * Y[j]));
      }
      dY[i] = s * winvd[i] * (f1 * r[i] + f2 * az);
    }
  }
  return L;
}

/* Loss of one sample and dL/dY. K: the plate's CSR (n = 2N rows). Returns L. */
double mp_loss(int N, const int* rp, const int* cols, const double* vals, const double* r, const double* e,
               const double* invd, double s, const double* Y, double* dY) {
  const long n = 2L * N;
  double c = 0.0, zaz = 0.0, er = 0.0;
  for (long i = 0; i < n; ++i) {
    const double zi = invd[i] * (r[i] + s * Y[i]);
    c += zi * r[i];
    er += e[i] * r[i];
    double az = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = cols[k];
      az += vals[k] * invd[j] * (r[j] + s * Y[j]);
    }
    zaz += zi * az;
  }
  const double L = 1.0 - c * c / (zaz * er);
  if (dY) {
    const double f1 = -2.0 * c / (zaz * er), f2 = 2.0 * c * c / (zaz * zaz * er);
    for (long i = 0; i < n; ++i) {
      double az = 0.0;
      for (int k = rp[i]; k < rp[i + 1]; ++k) {
        const int j = cols[k];
        az += vals[k] * invd[j] * (r[j] + s * Y[j]);
      }
      const double dz = f1 * r[i] + f2 * az;
      dY[i] = s * invd[i] * dz;
    }
  }
  return L;
}

/* Backward pass: adds dL/dP to dP, given the forward pass's H, G, A (from mp_forward with the
 * same q) and dY (N x 2). Work buffers: dH (N*F), dHn (N*F), dA (N*F). */
void mp_backward(int N, const int* node_ptr, const int* nbr, const double* X_in, const double* P, int q,
                 const double* H, const double* G, const double* A, const double* dY, double* dP,
                 double* dH, double* dHn, double* dA) {
  const long NF = (long)N * MP_F;
  const double* H3 = H + MP_L * NF;
  for (long i = 0; i < NF; ++i) dH[i] = 0.0;
  for (int n = 0; n < N; ++n)
    for (int c = 0; c < MP_OUT; ++c) {
      const double d = dY[(long)n * MP_OUT + c];
      dP[OFF_BOUT + c] += d;
      for (int k = 0; k < MP_F; ++k) {
        dP[OFF_WOUT + c * MP_F + k] += d * H3[(long)n * MP_F + k];
        dH[(long)n * MP_F + k] += d * P[OFF_WOUT + c * MP_F + k];
      }
    }
  for (int l = MP_L - 1; l >= 0; --l) {
    const double* Hp = H + l * NF;
    const double* Al = A + l * NF;
    const double* Gl = G + l * NF;
    const double* W = P + OFF_L0 + l * L_STRIDE;
    double* dW = dP + OFF_L0 + l * L_STRIDE;
    double* db = dW + MP_F * 2 * MP_F;
    for (long i = 0; i < NF; ++i) dHn[i] = dH[i];  /* residual path */
    for (int n = 0; n < N; ++n) {
      for (int k = 0; k < MP_F; ++k) dA[(long)n * MP_F + k] = 0.0;
      for (int o = 0; o < MP_F; ++o) {
        const double du = Gl[(long)n * MP_F + o] > 0.0 ? dH[(long)n * MP_F + o] : 0.0;
        if (du == 0.0) continue;
        db[o] += du;
        const double* w = W + o * 2 * MP_F;
        double* dw = dW + o * 2 * MP_F;
        for (int k = 0; k < MP_F; ++k) {
          dw[k] += du * Hp[(long)n * MP_F + k];
          dw[MP_F + k] += du * Al[(long)n * MP_F + k];
          dHn[(long)n * MP_F + k] += du * w[k];
          dA[(long)n * MP_F + k] += du * w[MP_F + k];
        }
      }
    }
    /* A_n = mean over neighbours: dH_{l-1,m} += dA_n / deg_n for each neighbour m of n */
    for (int n = 0; n < N; ++n) {
      int deg = 0;
      for (int k = node_ptr[n]; k < node_ptr[n + 1]; ++k) deg += nbr[k] != n;
      if (!deg) continue;
      for (int k = node_ptr[n]; k < node_ptr[n + 1]; ++k) {
        const int m = nbr[k];
        if (m == n) continue;
        for (int o = 0; o < MP_F; ++o) dHn[(long)m * MP_F + o] += dA[(long)n * MP_F + o] / deg;
      }
    }
    for (long i = 0; i < NF; ++i) dH[i] = dHn[i];
  }
  /* encoder: H0 = relu(W_in X + b_in) */
  for (int n = 0; n < N; ++n)
    for (int o = 0; o < MP_F; ++o) {
      const double du = H[(long)n * MP_F + o] > 0.0 ? dH[(long)n * MP_F + o] : 0.0;
      if (du == 0.0) continue;
      dP[OFF_BIN + o] += du;
      for (int k = 0; k < MP_IN; ++k) {
        const double xv = q ? rb(X_in[(long)n * MP_IN + k]) : X_in[(long)n * MP_IN + k];
        dP[OFF_WIN + o * MP_IN + k] += du * xv;
      }
    }
}
