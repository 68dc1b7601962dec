// Arguments shared by the fermion-operator kernel variants.
#pragma once
#include "common.cuh"

namespace susy {

template <typename R>
struct FopArgs {
  typedef typename CT<R>::T T;
  Geo g;
  const T* U;
  const T* Uinv;
  const T* pd;
  const T* src;
  T* dst;
  R G;
  int doG;
  const T* add;
  R addc;
  double* dot;
  const int* skip;  // device flag: nonzero = do nothing (finished solves)
  int comp_major;   // block order: 1 = all blocks of one output component together
  int nsb;          // site blocks per component
  const int* nbrtab;  // neighbour index table of the table-driven variant
  R eta_scale;        // 2 with the reference's RESCALE (the site component of
                      // input and output doubled, utilities.c:795,841), else 1
  T* trace;           // FOP_SITE_MAJOR_TR: the five traces Tr(U_e^-1 src_{1+e})
                      // of every site, [e][S] (written by its pre-pass)
};

constexpr int FOP_THREADS = 128;

// The three link indices not in {A, B}, ascending
template <int A, int B>
struct Compl {
  static constexpr int k(int n) {
    int c = 0;
    for (int v = 0; v < 5; v++) {
      if (v == A || v == B) continue;
      if (c == n) return v;
      c++;
    }
    return -1;
  }
  static constexpr int K0 = k(0), K1 = k(1), K2 = k(2);
};

}  // namespace susy
