// Analytic-potential tables held by a molecule handle (FP32 kernels of gto.cu).
#pragma once

#include <stdint.h>

namespace qmt {

// One merged primitive pair in FP32.
struct GPair32 {
  float px, py, pz;   // centre relative to the molecule's centroid (bohr)
  float p;            // exponent sum
  float fscale;       // sqrt(pi) / (2 sqrt(p)): far-field factor
  int L;
  int doff;           // offset of the pref * D_tuv coefficients
  int pad;
};

// One merged primitive pair in FP64: the off-site pairs that carry most of the charge.
struct GPair64 {
  double px, py, pz;  // centre relative to the molecule's centroid (bohr)
  double p;           // exponent sum
  double fscale;      // sqrt(pi) / (2 sqrt(p))
  int L;
  int doff;           // offset of the pref * D_tuv coefficients in dco64
};

// The FP32 tables of a molecule (device pointers).  Off-site pairs (two different atoms), sorted by
// L, are summed pair by pair; the pairs of one atom (centred on its nucleus) are kept per atom in
// descending exponent order with cumulative FP64 far-field moments, so that all of an atom's
// far-field pairs at a point are one FP64 multipole evaluation beside its nucleus.
struct Gto32Tables {
  const GPair32* pairs;     // off-site pairs evaluated in FP32, sorted by L
  int lstart[6];            // off-site pairs of angular momentum L: [lstart[L], lstart[L + 1])
  int slice[17];            // FP32 pair ranges of the nslice slices (equal estimated work)
  int nslice;
  const GPair64* pairs64;   // off-site pairs evaluated in FP64 (the largest charges), sorted by L
  int lstart64[6];
  int slice64[17];          // FP64 pair ranges of the nslice64 slices
  int nslice64;
  const double* dco64;      // their pref * D_tuv (double)
  const float* dco;         // pref * D_tuv of every FP32 pair (float)
  const GPair32* onsite;    // on-site pairs, atom by atom, descending exponent (`pad`: offset
                            // of their record in dco_on)
  const double* dco_on;     // on-site pair records: p, sqrt(pi) / (2 sqrt(p)), pref * D_tuv
  const float* onsite_p;    // their exponents (the same floats as onsite[i].p)
  const int* onsite_off;    // atom A's on-site pairs: [onsite_off[A], onsite_off[A + 1])
  const double* cum;        // per atom (m_A + 1) x 35: sum over its first k pairs of
                            // sqrt(pi) / (2 sqrt(p)) * pref * D_tuv (FP64), k = 0 .. m_A
  const int* cum_off;       // first row of atom A in cum
  const float* nuc;         // nuclei relative to the centroid (float x, y, z; the far / near test)
  const double* nuc64;      // the same in double
  double rx, ry, rz;        // the centroid
};

}  // namespace qmt
