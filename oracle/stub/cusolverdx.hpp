// cusolverdx.hpp -- a declarations-only stand-in for NVIDIA MathDx's
// cuSolverDx header, so that the reference's src/rbf_operators.h compiles for
// its host-callable fill code (PHS, PolyBasis, fill_matrix, fill_rhs).
//
// TEST INFRASTRUCTURE (oracle/ref_fill.cu only). It declares just the names
// the header's Solver / GESV / GELS alias templates and interp_config mention,
// as empty types; nothing here factors or solves, and no alias is ever
// instantiated. cuSolverDx itself is closed and absent from this build.
#pragma once

#define CUSOLVERDX_SKIP_IF_NOT_APPLICABLE_SM(solver)

namespace cusolverdx {

using byte = unsigned char;

enum class function { gesv_partial_pivot, gels };
enum class type { real, complex };
enum arrangement { col_major, row_major };

template <int M, int N, int K>
struct Size {};
template <function F>
struct Function {};
template <type Ty>
struct Type {};
template <typename T>
struct Precision {};
template <arrangement A, arrangement B>
struct Arrangement {};
template <int LD>
struct LeadingDimension {};
template <unsigned CC>
struct SM {};
struct Block {};

template <class A, class B>
struct Described {};
template <class A, class B>
Described<A, B> operator+(A, B) {
    return {};
}

namespace shared_memory {
template <class... Ts, class... Args>
void slice(byte* p, Args... args);
}  // namespace shared_memory

}  // namespace cusolverdx
