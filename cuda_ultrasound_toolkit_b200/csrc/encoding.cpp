// Transmit-encoding matrices (host side).
//
// Restates the upstream generator cuda_toolkit/src/rf_processing/hadamard/
// hadamard_decoder.cpp:110-222: Sylvester doubling H_2n = [[H, H], [H, -H]] from a
// base of order 1, 12 or 20, optionally re-ordered by sequency (WALSH). The order-12
// and order-20 bases are built from quadratic-residue characters (they equal the
// upstream tables at hadamard_decoder.cpp:8-45; see qr_base below).
//
// Besides the dense matrix (exported through cutb_encoding_matrix), the decode kernel
// needs the factorisation H_natural = S_{n/base} (x) B_base and the map from natural
// row to output row, which this file also provides.
#include "encoding.h"

#include <algorithm>
#include <numeric>

#include "common.cuh"

namespace cutb {

namespace {

// Order-12 and order-20 base matrices with a +1 border. With chi the quadratic
// character mod q (q = order - 1) and core indices a, b in [0, q):
//   order 12: core(a, b) = -1 if a == b, else chi(a - b)
//   order 20: core(a, b) = -1 if a + b == 0 mod q, else -chi(a + b)
std::vector<int8_t> qr_base(unsigned order)
{
    const unsigned q = order - 1;
    std::vector<int> chi(q, -1);
    chi[0] = 0;
    for (unsigned x = 1; x < q; ++x) chi[(x * x) % q] = 1;
    std::vector<int8_t> h(order * order, 1);
    for (unsigned i = 1; i < order; ++i)
        for (unsigned j = 1; j < order; ++j) {
            const unsigned a = i - 1, b = j - 1;
            int v;
            if (order == 12) v = a == b ? -1 : chi[(a + q - b) % q];
            else {
                const unsigned k = (a + b) % q;
                v = k == 0 ? -1 : -chi[k];
            }
            h[i * order + j] = (int8_t)v;
        }
    return h;
}

}  // namespace

bool build_encoding(unsigned n, int ordering, EncodingInfo& info)
{
    if (n == 0 || n > kMaxEncodingOrder) {
        set_error(CUTB_ERR_UNSUPPORTED, "Encoding order %u outside [1, %u].", n, kMaxEncodingOrder);
        return false;
    }
    if (ordering != HADAMARD && ordering != WALSH) {
        set_error(CUTB_ERR_UNSUPPORTED, "Encoding ordering %d is not HADAMARD or WALSH.", ordering);
        return false;
    }
    unsigned base;
    std::vector<int8_t> b;
    if (is_pow2(n)) { base = 1; b = {1}; }
    else if (n % 12 == 0 && is_pow2(n / 12)) { base = 12; b = qr_base(12); }
    else if (n % 20 == 0 && is_pow2(n / 20)) { base = 20; b = qr_base(20); }
    else {
        set_error(CUTB_ERR_UNSUPPORTED, "Encoding order %u not supported: only 2^n, 12*2^n or 20*2^n.", n);
        return false;
    }
    std::vector<int8_t> h((size_t)n * n, 0);
    for (unsigned i = 0; i < base; ++i)
        for (unsigned j = 0; j < base; ++j) h[(size_t)i * n + j] = b[i * base + j];
    for (unsigned len = base; len < n; len *= 2)
        for (unsigned r = 0; r < len; ++r)
            for (unsigned c = 0; c < len; ++c) {
                const int8_t v = h[(size_t)r * n + c];
                h[(size_t)r * n + c + len] = v;
                h[(size_t)(r + len) * n + c] = v;
                h[(size_t)(r + len) * n + c + len] = (int8_t)-v;
            }

    // Output row k holds natural row order[k]. WALSH sorts rows by their number of sign
    // changes with std::sort and upstream's comparator (hadamard_decoder.cpp:209-211), so rows
    // with equal counts (possible only with the 12/20 bases) land where upstream puts them.
    std::vector<unsigned> order(n);
    std::iota(order.begin(), order.end(), 0u);
    if (ordering == WALSH) {
        std::vector<unsigned> flips(n, 0);
        for (unsigned r = 0; r < n; ++r)
            for (unsigned c = 0; c + 1 < n; ++c)
                flips[r] += (h[(size_t)r * n + c] * h[(size_t)r * n + c + 1]) < 0;
        std::sort(order.begin(), order.end(), [&](unsigned x, unsigned y) { return flips[x] < flips[y]; });
    }

    info.n = n;
    info.base = base;
    info.matrix.resize((size_t)n * n);
    info.natural_to_output.resize(n);
    for (unsigned k = 0; k < n; ++k) {
        std::copy_n(h.begin() + (size_t)order[k] * n, n, info.matrix.begin() + (size_t)k * n);
        info.natural_to_output[order[k]] = (uint16_t)k;
    }
    return true;
}

}  // namespace cutb

extern "C" CUTB_API bool cutb_encoding_matrix(uint n, int ordering, signed char* out)
{
    CUTB_REQUIRE(out != nullptr, CUTB_ERR_INVALID_ARGUMENT, "cutb_encoding_matrix: null output.");
    cutb::EncodingInfo info;
    if (!cutb::build_encoding(n, ordering, info)) return false;
    std::copy(info.matrix.begin(), info.matrix.end(), out);
    return true;
}
