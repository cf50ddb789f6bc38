// One expansion order of the evaluator, compiled on its own: the build passes
// -DFMMB_P=<order> and links one object per order in FMMB_FOR_EACH_ORDER.
#include "evaluator_impl.cuh"

#ifndef FMMB_P
#error "FMMB_P (the expansion order) must be defined"
#endif

namespace fmmb {
template std::unique_ptr<EvaluatorBase> make_evaluator_at<FMMB_P>(bool, const EvaluatorArgs&, size_t*);
}  // namespace fmmb
