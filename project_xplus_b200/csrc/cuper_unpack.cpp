// cuper_unpack.cpp -- import of the reference's packed 16-channel Cuper stream
// (host/cuper_control_matrix.hpp:73-83 word layout, :130-207 channel/lane placement).
// Each 64-bit word is [63:50] local column, [49:32] packed row, [31:0] FP32 bits;
// packed rows with bit 17 set are padding.  The global row is restored from
// (channel, lane, packed_row) by inverting cuper_physical_pe_for_row
// (host/cuper_control_matrix.hpp:48-54), the same map the control kernel inverts at
// kernels/cuper_pcg_control_kernel.cpp:140-147.
#include <cstring>

#include "common.hpp"

namespace {
constexpr int kChannels = 16, kLanes = 8, kPe = kChannels * kLanes, kWindow = 8192;

inline int global_row(int channel, int lane, int packed_row) {
    const int checker = channel >> 1, acc = channel & 1;
    const int packet = (packed_row >> 1) * kPe + checker + acc * 8 + lane * 16;
    return packet * 2 + (packed_row & 1);
}
}  // namespace

using namespace xplus;

extern "C" int xplus_cuper_unpack(int n, int batch_count, const int* ptr, const uint64_t* words,
                                  int64_t channel_words, int64_t* nnz_out, int* rows, int* cols,
                                  float* vals) {
    return guarded([&] {
        require(n > 0 && batch_count > 0 && ptr && words && nnz_out, XPLUS_ERR_ARG, "invalid argument");
        require(static_cast<int64_t>(ptr[batch_count]) * kLanes <= channel_words, XPLUS_ERR_DATA,
                "packed stream shorter than sp_element_list_ptr says");
        int64_t count = 0;
        for (int b = 0; b < batch_count; ++b) {
            require(ptr[b] <= ptr[b + 1], XPLUS_ERR_DATA, "sp_element_list_ptr must be nondecreasing");
            for (int idx = ptr[b]; idx < ptr[b + 1]; ++idx)
                for (int c = 0; c < kChannels; ++c)
                    for (int l = 0; l < kLanes; ++l) {
                        const uint64_t w = words[static_cast<int64_t>(c) * channel_words + static_cast<int64_t>(idx) * kLanes + l];
                        const int prow = static_cast<int>((w >> 32) & 0x3FFFFull);
                        if (prow & (1 << 17)) continue;
                        const int col = b * kWindow + static_cast<int>((w >> 50) & 0x3FFFull);
                        const int row = global_row(c, l, prow);
                        require(row < n && col < n, XPLUS_ERR_DATA, "packed element outside the matrix");
                        if (rows) {
                            rows[count] = row;
                            cols[count] = col;
                            const uint32_t bits = static_cast<uint32_t>(w & 0xFFFFFFFFull);
                            std::memcpy(&vals[count], &bits, sizeof(float));
                        }
                        ++count;
                    }
        }
        *nnz_out = count;
    });
}
