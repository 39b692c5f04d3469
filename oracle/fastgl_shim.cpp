// Test infrastructure only: a C entry point over the reference's vendored fastgl
// (vendor/fastgl/fastgl.h:40-47), compiled together with that file into _ref/libfastgl_ref.so,
// so that tests can compare our Newton-based Gauss rule with the reference's rule.
#include <fastgl.h>

extern "C" int fastgl_rule(int n, double *x, double *w) {
    // nodal_basis.hpp:12-23: nodes[k-1] = -x_k, nodes[n-k] = x_k, k = 1..(n+1)/2
    for (int k = 1; k <= (n + 1) / 2; ++k) {
        auto pair = fastgl::GLPair(n, k);
        x[k - 1] = -pair.x();
        x[n - k] = pair.x();
        w[k - 1] = w[n - k] = pair.weight;
    }
    if (n % 2) x[n / 2] = 0;
    return 0;
}
