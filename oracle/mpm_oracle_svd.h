// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// 3x3 singular value decomposition A = U * diag(s) * V^T with U and V proper rotations and the
// sign of det(A) carried by s[2], which is the convention of the reference's svd3
// (include/math/svd3.h:1265-1276, the McAdams-Sifakis construction: Jacobi eigen-analysis of
// A^T A, column sort of B = A V, Givens QR of B).  This restatement follows the same three
// published steps (McAdams et al., "Computing the SVD of 3x3 matrices with minimal branching and
// elementary floating point operations", UW-Madison TR1690, 2011) but uses exact Jacobi and
// Givens rotations iterated to convergence instead of the paper's fixed-count approximate ones,
// so in double precision it is an accurate reference for the float kernels.
#pragma once

#include <cmath>
#include <utility>

namespace orc
{
    // Column-major 3x3: m[c * 3 + r].
    template <typename T>
    struct Svd3
    {
        T U[9], V[9], s[3];
    };

    template <typename T>
    inline void svd3(const T A[9], Svd3<T> &out)
    {
        auto at = [](const T *m, int r, int c) -> T { return m[c * 3 + r]; };
        // S = A^T A (symmetric).
        T S[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
            {
                T acc = 0;
                for (int k = 0; k < 3; ++k)
                    acc += at(A, k, i) * at(A, k, j);
                S[i][j] = acc;
            }
        T V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        // Cyclic Jacobi with exact rotations.
        const int maxSweeps = sizeof(T) == 4 ? 12 : 40;
        for (int sweep = 0; sweep < maxSweeps; ++sweep)
        {
            T off = S[0][1] * S[0][1] + S[0][2] * S[0][2] + S[1][2] * S[1][2];
            T diag = S[0][0] * S[0][0] + S[1][1] * S[1][1] + S[2][2] * S[2][2];
            if (off <= diag * (sizeof(T) == 4 ? T(1e-14) : T(1e-32)) || off == T(0))
                break;
            const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
            for (auto &pq : pairs)
            {
                int p = pq[0], q = pq[1];
                if (S[p][q] == T(0))
                    continue;
                T theta = (S[q][q] - S[p][p]) / (T(2) * S[p][q]);
                T t = (theta >= 0 ? T(1) : T(-1)) / (std::fabs(theta) + std::sqrt(theta * theta + T(1)));
                T c = T(1) / std::sqrt(t * t + T(1)), s = t * c;
                // S <- J^T S J with J the (p, q) rotation.
                for (int k = 0; k < 3; ++k)
                {
                    T skp = S[k][p], skq = S[k][q];
                    S[k][p] = c * skp - s * skq;
                    S[k][q] = s * skp + c * skq;
                }
                for (int k = 0; k < 3; ++k)
                {
                    T spk = S[p][k], sqk = S[q][k];
                    S[p][k] = c * spk - s * sqk;
                    S[q][k] = s * spk + c * sqk;
                }
                for (int k = 0; k < 3; ++k)
                {
                    T vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
        }
        // B = A V and sort columns by decreasing norm; every swap negates one column so that V
        // stays a proper rotation.
        T B[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                B[r][c] = at(A, r, 0) * V[0][c] + at(A, r, 1) * V[1][c] + at(A, r, 2) * V[2][c];
        auto colNorm2 = [&](int c) { return B[0][c] * B[0][c] + B[1][c] * B[1][c] + B[2][c] * B[2][c]; };
        auto swapCols = [&](int a, int b) {
            for (int r = 0; r < 3; ++r)
            {
                std::swap(B[r][a], B[r][b]);
                std::swap(V[r][a], V[r][b]);
                B[r][b] = -B[r][b];
                V[r][b] = -V[r][b];
            }
        };
        T n0 = colNorm2(0), n1 = colNorm2(1), n2 = colNorm2(2);
        if (n0 < n1) { swapCols(0, 1); std::swap(n0, n1); }
        if (n0 < n2) { swapCols(0, 2); std::swap(n0, n2); }
        if (n1 < n2) { swapCols(1, 2); std::swap(n1, n2); }
        // Givens QR: Q = U (rotation), R upper triangular with diag(R) = s.
        T U[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        const int rows[3][2] = {{0, 1}, {0, 2}, {1, 2}};
        const int cols[3] = {0, 0, 1};
        for (int g = 0; g < 3; ++g)
        {
            int p = rows[g][0], q = rows[g][1], col = cols[g];
            T a = B[p][col], b = B[q][col];
            T r = std::sqrt(a * a + b * b);
            T c = T(1), s = T(0);
            if (r > T(0))
            {
                c = a / r;
                s = b / r;
            }
            for (int k = 0; k < 3; ++k)
            {
                T bpk = B[p][k], bqk = B[q][k];
                B[p][k] = c * bpk + s * bqk;
                B[q][k] = -s * bpk + c * bqk;
            }
            // U <- U G^T
            for (int k = 0; k < 3; ++k)
            {
                T ukp = U[k][p], ukq = U[k][q];
                U[k][p] = c * ukp + s * ukq;
                U[k][q] = -s * ukp + c * ukq;
            }
        }
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
            {
                out.U[c * 3 + r] = U[r][c];
                out.V[c * 3 + r] = V[r][c];
            }
        out.s[0] = B[0][0];
        out.s[1] = B[1][1];
        out.s[2] = B[2][2];
    }
} // namespace orc
