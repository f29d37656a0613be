// TAGPU<T,Z>: drop-in replacement for the reference's TA<T,Z> (cpu/TA.h:10-38), the
// threshold algorithm over sorted attribute lists, running on a B200 through the C ABI
// in topk_b200.h.
//
// It derives from TPAcGPU (and so from the reference's own AA<T,Z>, cpu/AA.h:63-122),
// so the harness that drives TA (validation/bench_cpu.h:83-111) works after replacing
// the type:
//
//     TAGPU<float,uint64_t> ta(f.rows(), f.items());   // was TA<float,uint64_t>
//     f.gen(ta.get_cdata(), DISTR);  ta.init();  ta.findTopK(k, q, weights, attr);
//
// Behaviour: get_cdata() holds the table row-major (object i at cdata[i*d + m], as in
// TA); init() uploads it, transposes it on the device, runs the reference's normalize
// there (common/common.h:63-92, bit-exact), copies the normalised rows back into cdata
// and builds the sorted lists on the device (TA::init, cpu/TA.h:40-58).  findTopK is
// TA::findTopK (cpu/TA.h:61-96) on the device: it prints the same progress line, fills
// res ascending by score and sets threshold to the k-th score.  Each attribute is
// scored with its own weight; the reference reuses the weight of the list an object
// was found in (cpu/TA.h:83), so the two agree only when the queried weights are
// equal.  Ties at the k-th score go to the lower id.
#ifndef TOPK_B200_TAGPU_H
#define TOPK_B200_TAGPU_H

#include "topk_b200/TPAcGPU.h"

template <class T, class Z>
class TAGPU : public TPAcGPU<T, Z> {
 public:
  TAGPU(uint64_t n, uint64_t d, int device = 0) : TPAcGPU<T, Z>(n, d, device) { this->algo = "TAGPU"; }

  void init() {
    if (this->cdata == NULL) this->die(TOPK_ERR_STATE, "init() before the table was loaded into get_cdata()");
    this->check(topk_upload_rowmajor(this->handle(), this->cdata, this->d));
    this->check(topk_normalize(this->handle(), NULL, NULL));
    this->check(topk_download_rowmajor(this->handle(), this->cdata, this->d));
    this->t.start();
    this->check(topk_build_lists(this->handle()));
    this->tt_init = this->t.lap();
  }

  void findTopK(uint64_t k, uint8_t qq, T *weights, uint8_t *attr) {
    std::cout << this->algo << " find top-" << k << " (" << (int)qq << "D) ...";
    if (this->res.size() > 0) this->res.clear();
    const uint64_t c = k < this->n ? k : this->n;
    std::vector<uint64_t> ids(c);
    std::vector<float> scores(c);
    uint64_t count = 0, stats[3] = {0, 0, 0};
    float threshold = 0;
    this->t.start();
    this->check(topk_query_ta(this->handle(), k, qq, weights, attr, ids.data(), scores.data(), &count, &threshold,
                              stats));
    this->tt_processing += this->t.lap();
    if (STATS_EFF) this->tuple_count = stats[1];
    for (uint64_t j = 0; j < count; j++) this->res.push_back(tuple_<T, Z>((Z)ids[j], scores[j]));
    std::cout << std::fixed << std::setprecision(4);
    std::cout << " threshold=[" << threshold << "] (" << this->res.size() << ")" << std::endl;
    this->threshold = threshold;
  }
};

#endif  // TOPK_B200_TAGPU_H
