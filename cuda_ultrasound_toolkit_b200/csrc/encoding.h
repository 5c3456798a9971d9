// Transmit-encoding matrices: dense form plus the Kronecker factorisation used by
// the decode kernel.
#pragma once

#include <cstdint>
#include <vector>

namespace cutb {

// Largest encoding order accepted (upstream HADAMARD_MAX_SIZE, hadamard_decoder.cpp:6).
constexpr unsigned kMaxEncodingOrder = 1024;

struct EncodingInfo {
    unsigned n = 0;                       // order
    unsigned base = 1;                    // 1, 12 or 20: natural H = Sylvester(n / base) (x) base matrix
    std::vector<int8_t> matrix;           // n*n row-major, rows in output order
    std::vector<uint16_t> natural_to_output;  // natural (Kronecker) row index -> output row
};

// Builds the order-n matrix with HADAMARD (1) or WALSH (2) row order. Sets the error
// state and returns false for unsupported orders.
bool build_encoding(unsigned n, int ordering, EncodingInfo& info);

}  // namespace cutb
