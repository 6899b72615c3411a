/* Evaluates the functions of critmc_b200/csrc/fpmath.h on the host (compiled by the tests). */
#include "fpmath.h"
void cm_eval(int which, const float* x, const float* y, float* out, int n) {
  for (int i = 0; i < n; ++i) {
    float s, c;
    switch (which) {
      case 0: out[i] = cm_expf(x[i]); break;
      case 1: out[i] = cm_logf(x[i]); break;
      case 2: cm_sincosf(x[i], &s, &c); out[i] = s; break;
      case 3: cm_sincosf(x[i], &s, &c); out[i] = c; break;
      case 4: out[i] = cm_atan2f(y[i], x[i]); break;
      default: out[i] = cm_acosf(x[i]); break;
    }
  }
}
void cm_eval_d(const double* x, double* out, int n) {
  for (int i = 0; i < n; ++i) out[i] = cm_exp(x[i]);
}
void cm_eval_log_d(const double* x, double* out, int n) {
  for (int i = 0; i < n; ++i) out[i] = cm_log(x[i]);
}
