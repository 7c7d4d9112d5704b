// rh_bulk.h — layout of the FP32-bulk state.
//
// One oct of FP32-bulk state is one 192-byte record: rho, rho u, rho v, rho w
// of its 8 cells as float32 (cell fastest), then E of its 8 cells as float64.
// A state buffer holds the records back to back, so one bulk copy stages an
// oct.  Its float view uf and its double view ud (the buffer's doubles
// advanced by kBulkE, i.e. the first record's E) index oct o's values as
// uf[o * kBulkF + 8 * var + cell] and ud[o * kBulkD + cell].
#pragma once

namespace rh {

constexpr int kBulkF = 48;       // record stride in floats
constexpr int kBulkD = 24;       // record stride in doubles
constexpr int kBulkE = 16;       // doubles from a record's start to its E
constexpr int kBulkBytes = 192;  // bytes per record

}  // namespace rh
