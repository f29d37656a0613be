// TPArGPU<T,Z>: drop-in replacement for the reference's TPAr<T,Z> (cpu/TPAr.h:6-33),
// the row-major variant of the full-table evaluation, running on a B200 through the
// C ABI in topk_b200.h.
//
// It derives from TPAcGPU, which derives from the reference's own AA<T,Z>
// (cpu/AA.h:63-122), so a harness written for TPAr (validation/bench_cpu.h:113-152)
// works after replacing the type:
//
//     TPArGPU<float,uint64_t> tpar(f.rows(), f.items());   // was TPAr<float,uint64_t>
//     f.load(tpar.get_cdata());  tpar.init();  tpar.findTopKsimd(k, q, weights, attr);
//
// Behaviour: get_cdata() holds the table row-major (object i at cdata[i*d + m], as
// in TPAr); init() uploads it, transposes it on the device into the column-major
// table, runs the reference's normalize there (common/common.h:63-92, bit-exact: the
// same arithmetic per attribute as normalize_transpose) and copies the normalised
// rows back into cdata.  Queries are TPAcGPU's (exact, ties to the lower id), and
// unlike the reference's loops (8 or 16 objects per step with no tail) they read no
// object past n for any n.
#ifndef TOPK_B200_TPARGPU_H
#define TOPK_B200_TPARGPU_H

#include "topk_b200/TPAcGPU.h"

template <class T, class Z>
class TPArGPU : public TPAcGPU<T, Z> {
 public:
  TPArGPU(uint64_t n, uint64_t d, int device = 0) : TPAcGPU<T, Z>(n, d, device) { this->algo = "TPArGPU"; }

  void init() {
    if (this->cdata == NULL) this->die(TOPK_ERR_STATE, "init() before the table was loaded into get_cdata()");
    this->check(topk_upload_rowmajor(this->handle(), this->cdata, this->d));
    this->check(topk_normalize(this->handle(), NULL, NULL));
    this->check(topk_download_rowmajor(this->handle(), this->cdata, this->d));
    this->t.start();
    this->tt_init = this->t.lap();
  }
};

#endif  // TOPK_B200_TPARGPU_H
