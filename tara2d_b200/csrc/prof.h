// Per-kernel device timing: when enabled, an event is recorded on the
// launching stream before every kernel of a RHS evaluation and once at the
// end, so consecutive events bracket exactly one kernel.
#pragma once
#include <cuda_runtime.h>

namespace tara {

enum KernelKind : int {
  KK_COL_INV = 0,
  KK_ROW_COH,
  KK_COL_FWD_SIMPLE,
  KK_ROW_COM1,
  KK_COL_RT,
  KK_ROW_COM2,
  KK_COL_FWD_COM,
  KK_ROW_VORT,
  KK_COL_FWD_VORT,
  KK_ROW_FORCE,
  KK_CFL,
  KK_END,  // marks the end of the previous kernel
  KK_COUNT
};

inline const char* kernel_kind_name(int k) {
  static const char* n[KK_COUNT] = {"k_col_inv",      "k_row_coh",   "k_col_fwd_simple", "k_row_com1",
                                    "k_col_rt",       "k_row_com2",  "k_col_fwd_com",    "k_row_vort",
                                    "k_col_fwd_vort", "k_row_force", "k_cfl_update", "end"};
  return (k >= 0 && k < KK_COUNT) ? n[k] : "?";
}

struct Prof {
  int on = 0;
  int n = 0;
  int cap = 0;
  cudaEvent_t* ev = nullptr;
  int* kind = nullptr;
};

inline void prof_mark(Prof* p, cudaStream_t st, int kind) {
  if (!p || !p->on || p->n >= p->cap) return;
  cudaEventRecord(p->ev[p->n], st);
  p->kind[p->n] = kind;
  p->n++;
}

}  // namespace tara
