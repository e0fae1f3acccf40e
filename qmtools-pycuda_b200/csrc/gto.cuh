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

// The FP32 tables of a molecule (device pointers).  Off-site pairs (two different atoms), sorted by
// L, are summed pair by pair; the pairs of one atom (centred on its nucleus) are kept per atom in
// descending exponent order with cumulative FP64 far-field moments, so that all of an atom's
// far-field pairs at a point are one FP64 multipole evaluation beside its nucleus.
struct Gto32Tables {
  const GPair32* pairs;     // off-site pairs, sorted by L
  int lstart[6];            // off-site pairs of angular momentum L: [lstart[L], lstart[L + 1])
  int slice[17];            // off-site pair ranges of the nslice slices (equal estimated work)
  int nslice;
  const float* dco;         // pref * D_tuv of every pair (float)
  const GPair32* onsite;    // on-site pairs, atom by atom, descending exponent
  const float* onsite_p;    // their exponents (the same floats as onsite[i].p)
  const int* onsite_off;    // atom A's on-site pairs: [onsite_off[A], onsite_off[A + 1])
  const double* cum;        // per atom (m_A + 1) x 35: sum over its first k pairs of
                            // sqrt(pi) / (2 sqrt(p)) * pref * D_tuv (FP64), k = 0 .. m_A
  const int* cum_off;       // first row of atom A in cum
  const float* nuc;         // nuclei relative to the centroid (float x, y, z)
  double rx, ry, rz;        // the centroid
};

}  // namespace qmt
