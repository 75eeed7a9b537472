// grav_dft.cu -- split-BF16 DFT-as-GEMM gravity solve (tcgen05). Not built
// yet: plans of this precision report TPT_ERR_UNSUPPORTED.
#include "grav_dft.hpp"

namespace tpt {
namespace dft {

struct DftImpl {
    std::vector<JobShape> shapes;
};

int DftSet::create(const std::vector<JobShape> &shapes) {
    (void)shapes;
    TPT_FAIL(TPT_ERR_UNSUPPORTED, "split-BF16 gravity is not available in this build");
}
void DftSet::dims(size_t, uint32_t *n1, uint32_t *n2) const {
    *n1 = 0;
    *n2 = 0;
}
int DftSet::set_io(size_t, const SolveIO &) { TPT_FAIL(TPT_ERR_UNSUPPORTED, "split-BF16 gravity unavailable"); }
int DftSet::launch(cudaStream_t, const SolveIO *) const {
    TPT_FAIL(TPT_ERR_UNSUPPORTED, "split-BF16 gravity unavailable");
}
uint32_t DftSet::launches() const { return 0; }
double DftSet::flops() const { return 0.0; }
void DftSet::destroy() {
    delete impl;
    impl = nullptr;
}

}  // namespace dft
}  // namespace tpt
