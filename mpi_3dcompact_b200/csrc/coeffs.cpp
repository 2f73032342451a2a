// Host-side set-up of the compact operators: RHS stencils, boundary closures
// and the LU factors of the (cyclic) banded left-hand sides, all in FP64.
//
// The factors are produced by the same elimination sequence the reference
// runs on every call (src/Utils.cpp:4-191), once per operator instead of once
// per line: the GPU line solve then only replays the RHS-dependent half.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "mc3d_internal.h"

namespace mc3d {

namespace {

// Thomas factorisation of src/Utils.cpp:4-20: work[] and the multipliers m[].
void tri_factor(const std::vector<double> &a, const std::vector<double> &b, const std::vector<double> &c,
                std::vector<double> &m, std::vector<double> &work) {
    int n = (int)b.size();
    work = b;
    m.assign(n, 0.0);
    for (int ip = 1; ip < n; ip++) {
        m[ip] = a[ip] / work[ip - 1];
        work[ip] = work[ip] - m[ip] * c[ip - 1];
    }
}

// Full solveTri (src/Utils.cpp:4-20) for set-up vectors.
std::vector<double> tri_solve(const std::vector<double> &a, const std::vector<double> &b,
                              const std::vector<double> &c, const std::vector<double> &d) {
    int n = (int)b.size();
    std::vector<double> work = b, x = d;
    for (int ip = 1; ip < n; ip++) {
        double m = a[ip] / work[ip - 1];
        work[ip] = work[ip] - m * c[ip - 1];
        x[ip] = x[ip] - m * x[ip - 1];
    }
    x[n - 1] /= work[n - 1];
    for (int ip = n - 2; ip >= 0; ip--) x[ip] = (x[ip] - c[ip] * x[ip + 1]) / work[ip];
    return x;
}

// Matrix half of solvePenta (src/Utils.cpp:48-83): multipliers m1 (row ip,
// column ip-1), m2 (row ip+1, column ip-1), mL, and the final C and D.
struct PentaFactor {
    std::vector<double> m1, m2, C, D;
    double mL;
};
PentaFactor penta_factor(const std::vector<double> &e, const std::vector<double> &a, const std::vector<double> &d,
                         const std::vector<double> &c, const std::vector<double> &f) {
    int size = (int)d.size();
    PentaFactor P;
    std::vector<double> x = a, C = c, D = d;
    P.m1.assign(size, 0.0);
    P.m2.assign(size, 0.0);
    for (int ip = 1; ip < size - 1; ip++) {
        double xm = x[ip - 1] / D[ip - 1];
        P.m1[ip] = xm;
        D[ip] = D[ip] - xm * C[ip - 1];
        C[ip] = C[ip] - xm * f[ip - 1];
        xm = e[ip - 1] / D[ip - 1];
        P.m2[ip] = xm;
        x[ip] = x[ip] - xm * C[ip - 1];
        D[ip + 1] = D[ip + 1] - xm * f[ip - 1];
    }
    P.mL = x[size - 2] / D[size - 2];
    D[size - 1] = D[size - 1] - P.mL * C[size - 2];
    P.C = C;
    P.D = D;
    return P;
}

// Full solvePenta for set-up vectors (same arithmetic order as the reference).
std::vector<double> penta_solve(const std::vector<double> &e, const std::vector<double> &a,
                                const std::vector<double> &d, const std::vector<double> &c,
                                const std::vector<double> &f, const std::vector<double> &b) {
    int size = (int)d.size();
    std::vector<double> x = a, B = b, C = c, D = d;
    for (int ip = 1; ip < size - 1; ip++) {
        double xm = x[ip - 1] / D[ip - 1];
        D[ip] = D[ip] - xm * C[ip - 1];
        C[ip] = C[ip] - xm * f[ip - 1];
        B[ip] = B[ip] - xm * B[ip - 1];
        xm = e[ip - 1] / D[ip - 1];
        x[ip] = x[ip] - xm * C[ip - 1];
        D[ip + 1] = D[ip + 1] - xm * f[ip - 1];
        B[ip + 1] = B[ip + 1] - xm * B[ip - 1];
    }
    double xm = x[size - 2] / D[size - 2];
    D[size - 1] = D[size - 1] - xm * C[size - 2];
    std::vector<double> out(size);
    out[size - 1] = (B[size - 1] - xm * B[size - 2]) / D[size - 1];
    out[size - 2] = (B[size - 2] - C[size - 2] * out[size - 1]) / D[size - 2];
    for (int ip = size - 3; ip >= 0; ip--)
        out[ip] = (B[ip] - f[ip] * out[ip + 2] - C[ip] * out[ip + 1]) / D[ip];
    return out;
}

double minor3(const double m[16], int r0, int r1, int r2, int c0, int c1, int c2) {
    return m[4 * r0 + c0] * (m[4 * r1 + c1] * m[4 * r2 + c2] - m[4 * r2 + c1] * m[4 * r1 + c2]) -
           m[4 * r0 + c1] * (m[4 * r1 + c0] * m[4 * r2 + c2] - m[4 * r2 + c0] * m[4 * r1 + c2]) +
           m[4 * r0 + c2] * (m[4 * r1 + c0] * m[4 * r2 + c1] - m[4 * r2 + c0] * m[4 * r1 + c1]);
}

// 4x4 inverse by adjugate over determinant (the method of src/Utils.cpp:193-224).
void inverse4(const double m[16], double inv[16]) {
    const int R[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            // cofactor of element (j, i), transposed into inv[i][j]
            double mn = minor3(m, R[j][0], R[j][1], R[j][2], R[i][0], R[i][1], R[i][2]);
            inv[4 * i + j] = ((i + j) % 2 ? -mn : mn);
        }
    double det = m[0] * minor3(m, 1, 2, 3, 1, 2, 3) - m[1] * minor3(m, 1, 2, 3, 0, 2, 3) +
                 m[2] * minor3(m, 1, 2, 3, 0, 1, 3) - m[3] * minor3(m, 1, 2, 3, 0, 1, 2);
    double id = 1.0 / det;
    for (int i = 0; i < 16; i++) inv[i] *= id;
}

// Packed factor layout (LineOpHost::arr), N values per array:
//   tri:   [m | rw | c | z]          (z only for the cyclic kind)
//   penta: [m1 | m2 | rD | C | f | z0 | z1 | z2 | z3]  (z* only cyclic)
void pack_tri(LineOpHost &op, const std::vector<double> &a, const std::vector<double> &b,
              const std::vector<double> &c, bool cyclic, double alpha, double beta) {
    int n = op.N;
    std::vector<double> bb = b;
    double gamma = 0;
    if (cyclic) {   // src/Utils.cpp:22-46
        gamma = -b[0];
        bb[0] = b[0] - gamma;
        bb[n - 1] = b[n - 1] - alpha * beta / gamma;
    }
    std::vector<double> m, work;
    tri_factor(a, bb, c, m, work);
    op.arr.assign(4 * n, 0.0);
    for (int i = 0; i < n; i++) {
        op.arr[i] = m[i];
        op.arr[n + i] = 1.0 / work[i];
        op.arr[2 * n + i] = c[i];
    }
    if (cyclic) {
        std::vector<double> u(n, 0.0);
        u[0] = gamma;
        u[n - 1] = alpha;
        std::vector<double> z = tri_solve(a, bb, c, u);
        for (int i = 0; i < n; i++) op.arr[3 * n + i] = z[i];
        op.sc[0] = beta;
        op.sc[1] = 1.0 / gamma;
        op.sc[2] = 1.0 / (1.0 + z[0] + beta * z[n - 1] / gamma);
    }
}

void pack_penta(LineOpHost &op, const std::vector<double> &lo2, const std::vector<double> &lo,
                const std::vector<double> &dg, const std::vector<double> &up, const std::vector<double> &up2,
                bool cyclic, const double cp[6]) {
    int n = op.N;
    PentaFactor P = penta_factor(lo2, lo, dg, up, up2);
    op.arr.assign(9 * n, 0.0);
    for (int i = 0; i < n; i++) {
        op.arr[i] = P.m1[i];
        op.arr[n + i] = P.m2[i];
        op.arr[2 * n + i] = 1.0 / P.D[i];
        op.arr[3 * n + i] = P.C[i];
        op.arr[4 * n + i] = up2[i];
    }
    op.arr[n - 1] = P.mL;   // row N-1 uses mL in place of m1
    if (cyclic) {           // Woodbury set-up of src/Utils.cpp:85-157
        std::vector<std::vector<double> > Z(4), V(4, std::vector<double>(n, 0.0));
        int upos[4] = {0, 1, n - 2, n - 1};
        for (int j = 0; j < 4; j++) {
            std::vector<double> u(n, 0.0);
            u[upos[j]] = 1.0;
            Z[j] = penta_solve(lo2, lo, dg, up, up2, u);
        }
        V[0][n - 2] = cp[0];
        V[0][n - 1] = cp[1];
        V[1][n - 1] = cp[2];
        V[2][0] = cp[3];
        V[3][0] = cp[4];
        V[3][1] = cp[5];
        double Pm[16];
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) {
                double s = 0.0;
                for (int k = 0; k < n; k++) s += V[i][k] * Z[j][k];
                Pm[4 * i + j] = s + (i == j ? 1.0 : 0.0);
            }
        inverse4(Pm, op.Hm);
        for (int j = 0; j < 4; j++)
            for (int i = 0; i < n; i++) op.arr[(5 + j) * n + i] = Z[j][i];
        for (int i = 0; i < 6; i++) op.cp[i] = cp[i];
    }
}

}  // namespace

LineOpHost build_deriv_op(int fd_type, int bc_type, int N, double dh) {
    if (N <= 10) throw std::runtime_error("line length must be greater than 10 (src/Options.cpp:241-244)");
    LineOpHost op;
    op.N = N;
    op.deriv = true;
    op.inv_dh = 1.0 / dh;
    bool per = bc_type == MC3D_PERIODIC_SOLVE;
    if (fd_type == MC3D_PADE6) {
        // src/Pade6.hpp:70-75 interior, :78-137 boundary scheme 1, :183-215 bands
        double alpha = 1.0 / 3.0, a = 14.0 / 9.0, b = 1.0 / 9.0;
        op.H = 2;
        op.st[0] = -b / 4.0;
        op.st[1] = -a / 2.0;
        op.st[3] = a / 2.0;
        op.st[4] = b / 4.0;
        std::vector<double> lo(N, alpha), up(N, alpha), dg(N, 1.0);
        if (per) {
            op.kind = K_TRI_PER;
            pack_tri(op, lo, dg, up, true, alpha, alpha);
        } else {
            op.kind = K_TRI_DIR;
            double alpha11 = 2.0, alpha21 = 1.0 / 6.0, alpha22 = 1.0 / 2.0;
            up[0] = alpha11; up[1] = alpha22; lo[1] = alpha21;
            lo[N - 1] = alpha11; lo[N - 2] = alpha22; up[N - 2] = alpha21;
            double a1 = -5.0 / 2.0, b1 = 2.0, c1 = 1.0 / 2.0;
            double a2 = -5.0 / 9.0, b2 = -1.0 / 2.0, c2 = 1.0, d2 = 1.0 / 18.0;
            op.bw = 6;
            op.head = {a1, b1, c1, 0.0, 0.0, 0.0, a2, b2, c2, d2, 0.0, 0.0};
            // rows N-1 and N-2 are the mirrored, negated closures (src/Pade6.cpp:306-310)
            op.tail = {0.0, 0.0, 0.0, -c1, -b1, -a1,    // row N-1 on phi[N-6..N-1]
                       0.0, 0.0, -d2, -c2, -b2, -a2};  // row N-2
            pack_tri(op, lo, dg, up, false, 0, 0);
        }
    } else if (fd_type == MC3D_PENTA10) {
        // src/Penta10.hpp:68-175
        double beta = 1.0 / 20.0, alpha = 1.0 / 2.0, a = 17.0 / 12.0, b = 101.0 / 150.0, c = 1.0 / 100.0;
        op.H = 3;
        op.st[0] = -c / 6.0; op.st[1] = -b / 4.0; op.st[2] = -a / 2.0;
        op.st[4] = a / 2.0;  op.st[5] = b / 4.0;  op.st[6] = c / 6.0;
        std::vector<double> dg(N, 1.0), lo(N, alpha), up(N, alpha), lo2(N, beta), up2(N, beta);
        if (per) {
            op.kind = K_PEN_PER;
            double cp[6] = {beta, alpha, beta, beta, alpha, beta};
            pack_penta(op, lo2, lo, dg, up, up2, true, cp);
        } else {
            op.kind = K_PEN_DIR;
            double beta1 = 0.0, alpha1 = 5.0;
            double beta2 = 0.0, alpha2_1 = 1.0 / 12.0, alpha2_2 = 5.0 / 4.0;
            double beta3_1 = 1.0 / 36.0, beta3_2 = 1.0 / 36.0, alpha3_1 = 4.0 / 9.0, alpha3_2 = 4.0 / 9.0;
            up[0] = alpha1; up[1] = alpha2_2; up[2] = alpha3_2;
            lo[0] = alpha2_1; lo[1] = alpha3_1;
            up2[0] = beta1; up2[1] = beta2; up2[2] = beta3_2;
            lo2[0] = beta3_1;
            up[N - 2] = alpha2_1; up[N - 3] = alpha3_1;
            lo[N - 2] = alpha1; lo[N - 3] = alpha2_2; lo[N - 4] = alpha3_2;
            up2[N - 3] = beta3_1;
            lo2[N - 3] = beta1; lo2[N - 4] = beta2; lo2[N - 5] = beta3_2;
            double r1[9] = {-197.0 / 60.0, -5.0 / 12.0, 5.0, -5.0 / 3.0, 5.0 / 12.0, -1.0 / 20.0, 0, 0, 0};
            double r2[9] = {-79.0 / 240.0, -77.0 / 60.0, 55.0 / 48.0, 5.0 / 9.0, -5.0 / 48.0, 1.0 / 60.0,
                            -1.0 / 720.0, 0.0, 0.0};
            double r3[9] = {-25.0 / 54.0 / 4.0, -40.0 / 27.0 / 2.0, 0.0, 40.0 / 27.0 / 2.0, 25.0 / 54.0 / 4.0,
                            0.0, 0.0, 0.0, 0.0};
            op.bw = 9;
            op.head.assign(3 * 9, 0.0);
            op.tail.assign(3 * 9, 0.0);
            const double *rows[3] = {r1, r2, r3};
            for (int r = 0; r < 3; r++)
                for (int k = 0; k < 9; k++) {
                    op.head[r * 9 + k] = rows[r][k];
                    // row N-1-r on phi[N-9..N-1]: coefficient of phi[N-1-k] is -rows[r][k]
                    op.tail[r * 9 + (8 - k)] = -rows[r][k];
                }
            double cp[6] = {0, 0, 0, 0, 0, 0};
            pack_penta(op, lo2, lo, dg, up, up2, false, cp);
        }
    } else if (fd_type == MC3D_CD2) {
        // src/CD2.hpp:56-63 and src/CD2.cpp:129-183: interior row is
        // (a*phi[i+1] + c*phi[i-1])/h with a = -1/2, c = 1/2 (sign as the reference)
        op.H = 1;
        op.st[0] = 0.5;
        op.st[2] = -0.5;
        if (per) {
            op.kind = K_EXPL_PER;
        } else {
            op.kind = K_EXPL_DIR;
            op.bw = 3;
            op.head = {-1.5, 2.0, -0.5};
            op.tail = {-0.5, 2.0, -1.5};   // (aa*phi[N-1] + bb*phi[N-2] + cc*phi[N-3])
        }
    } else {
        throw std::runtime_error("unknown derivative type");
    }
    return op;
}

LineOpHost build_filter_op(int filter_type, double af, int bc_type, int N) {
    if (N <= 10) throw std::runtime_error("line length must be greater than 10 (src/Options.cpp:241-244)");
    LineOpHost op;
    op.N = N;
    op.deriv = false;
    op.inv_dh = 1.0;
    bool per = bc_type == MC3D_PERIODIC_SOLVE;
    std::vector<double> a;
    std::vector<std::vector<double> > fb;
    if (filter_type == MC3D_COMPACT10) {
        // src/Compact10Filter.hpp:58-134 (boundary scheme 1)
        a = {(193.0 + 126.0 * af) / 256.0, (105.0 + 302.0 * af) / 256.0, (-15.0 + 30.0 * af) / 64.0,
             (45.0 - 90.0 * af) / 512.0, (-5.0 + 10.0 * af) / 256.0, (1.0 - 2.0 * af) / 512.0};
        fb = {{(1.0 + 1022.0 * af) / 1024.0, (507.0 + 10.0 * af) / 512.0, (45.0 + 934.0 * af) / 1024.0,
               (-15.0 + 30.0 * af) / 128.0, (105.0 - 210.0 * af) / 512.0, (-63.0 + 126.0 * af) / 256.0,
               (105.0 - 210.0 * af) / 512.0, (-15.0 + 30.0 * af) / 128.0, (45.0 - 90.0 * af) / 1024.0,
               (-5.0 + 10.0 * af) / 512.0, (1.0 - 2.0 * af) / 1024.0},
              {(-1.0 + 2.0 * af) / 1024.0, (5.0 + 502.0 * af) / 512.0, (979.0 + 90.0 * af) / 1024.0,
               (15.0 + 98.0 * af) / 128.0, (-105.0 + 210.0 * af) / 512.0, (63.0 - 126.0 * af) / 256.0,
               (-105.0 + 210.0 * af) / 512.0, (15.0 - 30.0 * af) / 128.0, (-45.0 + 90.0 * af) / 1024.0,
               (5.0 - 10.0 * af) / 512.0, (-1.0 + 2.0 * af) / 1024.0},
              {(1.0 - 2.0 * af) / 1024.0, (-5.0 + 10.0 * af) / 512.0, (45.0 + 934.0 * af) / 1024.0,
               (113.0 + 30.0 * af) / 128.0, (105.0 + 302.0 * af) / 512.0, (-63.0 + 126.0 * af) / 256.0,
               (105.0 - 210.0 * af) / 512.0, (-15.0 + 30.0 * af) / 128.0, (45.0 - 90.0 * af) / 1024.0,
               (-5.0 + 10.0 * af) / 512.0, (1.0 - 2.0 * af) / 1024.0},
              {(-1.0 + 2.0 * af) / 1024.0, (5.0 - 10.0 * af) / 512.0, (-45.0 + 90.0 * af) / 1024.0,
               (15.0 + 98.0 * af) / 128.0, (407.0 + 210.0 * af) / 512.0, (63.0 + 130.0 * af) / 256.0,
               (-105.0 + 210.0 * af) / 512.0, (15.0 - 30.0 * af) / 128.0, (-45.0 + 90.0 * af) / 1024.0,
               (5.0 - 10.0 * af) / 512.0, (-1.0 + 2.0 * af) / 1024.0}};
    } else if (filter_type == MC3D_COMPACT8) {
        // src/Compact8Filter.hpp:55-94
        a = {(93.0 + 70.0 * af) / 128.0, (7.0 + 18.0 * af) / 16.0, (-7.0 + 14.0 * af) / 32.0,
             (1.0 - 2.0 * af) / 16.0, (-1.0 + 2.0 * af) / 128.0};
        fb = {{1.0 / 256.0 + 127.0 * af / 128.0, 31.0 / 32.0 + 1.0 * af / 16.0, 7.0 / 64.0 + 25.0 * af / 32.0,
               -7.0 / 32.0 + 7.0 * af / 16.0, 7.0 * (5.0 - 10.0 * af) / 128.0, -7.0 / 32.0 + 7.0 * af / 16.0,
               7.0 / 64.0 - 7.0 * af / 32.0, -1.0 / 32.0 + 1.0 * af / 16.0, 1.0 / 256.0 - 1.0 * af / 128.0},
              {-1.0 / 256.0 + 1.0 * af / 128.0, 1.0 / 32.0 + 15.0 * af / 16.0, 57.0 / 64.0 + 7.0 * af / 32.0,
               7.0 / 32.0 + 9.0 * af / 16.0, 7.0 * (-5.0 + 10.0 * af) / 128.0, 7.0 / 32.0 - 7.0 * af / 16.0,
               -7.0 / 64.0 + 7.0 * af / 32.0, 1.0 / 32.0 - 1.0 * af / 16.0, -1.0 / 256.0 + 1.0 * af / 128.0},
              {1.0 / 256.0 - 1.0 * af / 128.0, -1.0 / 32.0 + 1.0 * af / 16.0, 7.0 / 64.0 + 25.0 * af / 32.0,
               25.0 / 32.0 + 7.0 * af / 16.0, 35.0 / 128.0 + 29.0 * af / 64.0, -7.0 / 32.0 + 7.0 * af / 16.0,
               7.0 / 64.0 - 7.0 * af / 32.0, -1.0 / 32.0 + 1.0 * af / 16.0, 1.0 / 256.0 - 1.0 * af / 128.0}};
    } else {
        throw std::runtime_error("unknown filter type");
    }
    int H = (int)a.size() - 1;
    op.H = H;
    // symmetric interior stencil (src/Compact10Filter.cpp:5-75): cc0 = a0, cck = ak/2
    for (int k = -H; k <= H; k++) op.st[k + H] = (k == 0) ? a[0] : a[k < 0 ? -k : k] / 2.0;
    std::vector<double> lo(N, af), up(N, af), dg(N, 1.0);
    if (per) {
        op.kind = K_TRI_PER;
        pack_tri(op, lo, dg, up, true, af, af);
    } else {
        op.kind = K_TRI_DIR;
        lo[0] = up[0] = lo[N - 1] = up[N - 1] = 0.0;
        int bw = (int)fb[0].size();
        op.bw = bw;
        op.head.assign(H * bw, 0.0);
        op.tail.assign(H * bw, 0.0);
        op.head[0] = 1.0;                  // RHSvec[0] = phi[0]
        op.tail[bw - 1] = 1.0;             // RHSvec[N-1] = phi[N-1]
        for (int r = 1; r < H; r++)
            for (int k = 0; k < bw; k++) {
                op.head[r * bw + k] = fb[r - 1][k];
                op.tail[r * bw + (bw - 1 - k)] = fb[r - 1][k];   // mirrored on phi[N-1-k]
            }
        pack_tri(op, lo, dg, up, false, 0, 0);
    }
    return op;
}

// DSM test filters (src/CommN5PadeTestFilter.{hpp,cpp}, src/CommN5ExpTestFilter.{hpp,cpp}).
// MC3D_TESTFILTER_PADE: 11-point RHS, pentadiagonal LHS (v2, 0, v0, 0, v2),
// cyclic or with nodes 0..4 / N-5..N-1 explicitly filtered; MC3D_TESTFILTER_EXP:
// explicit 7-point filter. Both share the one-sided closures of nodes 0..2.
LineOpHost build_testfilter_op(int type, int bc_type, int N) {
    if (N <= 10) throw std::runtime_error("line length must be greater than 10 (src/Options.cpp:241-244)");
    static const double B[3][6] = {{31.0 / 32.0, 5.0 / 32.0, -5.0 / 16.0, 5.0 / 16.0, -5.0 / 32.0, 1.0 / 32.0},
                                   {1.0 / 32.0, 27.0 / 32.0, 5.0 / 16.0, -5.0 / 16.0, 5.0 / 32.0, -1.0 / 32.0},
                                   {-1.0 / 32.0, 5.0 / 32.0, 11.0 / 16.0, 5.0 / 16.0, -5.0 / 32.0, 1.0 / 32.0}};
    static const double w[4] = {11.0 / 16.0, 15.0 / 64.0, -3.0 / 32.0, 1.0 / 64.0};
    static const double wi[6] = {7.0 / 24.0, 175.0 / 768.0, 5.0 / 48.0, 35.0 / 1536.0, 0.0, -1.0 / 1536.0};
    const double v0 = 7.0 / 12.0, v1 = 0.0, v2 = 5.0 / 24.0;
    LineOpHost op;
    op.N = N;
    op.deriv = false;
    op.inv_dh = 1.0;
    const bool per = bc_type == MC3D_PERIODIC_SOLVE;
    // head row r on phi[0..bw-1]; tail row r (node N-1-r) mirrored onto phi[N-bw..N-1]
    auto closures = [&](int H, int bw) {
        op.bw = bw;
        op.head.assign(H * bw, 0.0);
        op.tail.assign(H * bw, 0.0);
        for (int r = 0; r < 3; r++)
            for (int k = 0; k < 6; k++) {
                op.head[r * bw + k] = B[r][k];
                op.tail[r * bw + (bw - 1 - k)] = B[r][k];
            }
    };
    if (type == MC3D_TESTFILTER_EXP) {
        op.H = 3;
        for (int k = -3; k <= 3; k++) op.st[k + 3] = w[k < 0 ? -k : k];
        if (per) {
            op.kind = K_EXPL_PER;
        } else {
            op.kind = K_EXPL_DIR;
            closures(3, 6);
        }
        return op;
    }
    if (type != MC3D_TESTFILTER_PADE) throw std::runtime_error("unknown test filter type");
    op.H = 5;
    for (int k = -5; k <= 5; k++) op.st[k + 5] = wi[k < 0 ? -k : k];
    std::vector<double> dg(N, v0), lo(N, v1), up(N, v1), lo2(N, v2), up2(N, v2);
    if (per) {
        op.kind = K_PEN_PER;
        const double cp[6] = {v2, v1, v2, v2, v1, v2};
        pack_penta(op, lo2, lo, dg, up, up2, true, cp);
        return op;
    }
    op.kind = K_PEN_DIR;
    // nodes 0..4 and N-5..N-1: identity rows (CommN5PadeTestFilter.hpp:83-177)
    for (int r = 0; r < 5; r++) {
        dg[r] = dg[N - 1 - r] = 1.0;
        up[r] = up2[r] = 0.0;
    }
    for (int i = 0; i < 4; i++) lo[i] = 0.0;
    for (int i = 0; i < 3; i++) lo2[i] = 0.0;
    for (int i = N - 7; i < N - 2; i++) lo2[i] = 0.0;
    for (int i = N - 6; i < N - 1; i++) lo[i] = 0.0;
    for (int i = N - 5; i < N - 1; i++) up[i] = 0.0;
    for (int i = N - 5; i < N - 2; i++) up2[i] = 0.0;
    closures(5, 8);
    // nodes 3, 4: 7-point rows on phi[r-3..r+3] (CommN5PadeTestFilter.cpp:106-111, :125-130)
    for (int r = 3; r < 5; r++)
        for (int s = -3; s <= 3; s++) {
            const double c = w[s < 0 ? -s : s];
            op.head[r * 8 + (r + s)] = c;
            op.tail[r * 8 + (7 - (r + s))] = c;
        }
    const double cp0[6] = {0, 0, 0, 0, 0, 0};
    pack_penta(op, lo2, lo, dg, up, up2, false, cp0);
    return op;
}

namespace {
// Stationary interior of the factor arrays (equality after rounding to the
// working precision) and the correction window.
void analyse(LineOpHost &h, int precision) {
    int n = h.N;
    size_t na = h.arr.size() / (n ? n : 1);
    int nfac = h.kind == K_TRI_PER || h.kind == K_TRI_DIR ? 3 : (h.kind == K_PEN_PER || h.kind == K_PEN_DIR ? 5 : 0);
    const bool f32 = precision != MC3D_FP64;
    h.stat_lo = h.stat_hi = 0;
    if (nfac && na >= (size_t)nfac) {
        // largest run [lo, hi) with all factor arrays (and a1[n-1]) constant
        auto at = [&](int a, int i) {
            double v = h.arr[(size_t)a * n + i];
            return f32 ? (double)(float)v : v;
        };
        int best_lo = 0, best_hi = 0, lo = 1;
        for (int i = 1; i < n; i++) {
            bool same = true;
            for (int a = 0; a < nfac && same; a++) same = at(a, i) == at(a, lo);
            same = same && at(1, i - 1) == at(1, lo);
            if (!same) lo = i;
            if (i + 1 - lo > best_hi - best_lo) { best_lo = lo; best_hi = i + 1; }
        }
        if (best_hi - best_lo >= 16 && best_lo >= 2) {
            h.stat_lo = best_lo;
            h.stat_hi = best_hi;
            for (int a = 0; a < nfac; a++) h.stat_c[a] = at(a, best_lo);
        }
    }
    h.corr_lo = h.corr_hi = 0;
    int first = -1, ncol = h.kind == K_TRI_PER ? 1 : (h.kind == K_PEN_PER ? 4 : 0);
    if (ncol) {
        int base = h.kind == K_TRI_PER ? 3 : 5;
        double peak = 0;
        for (int c = 0; c < ncol; c++)
            for (int i = 0; i < n; i++) peak = std::max(peak, std::fabs(h.arr[(size_t)(base + c) * n + i]));
        const double thr = peak * std::ldexp(1.0, f32 ? -32 : -64);
        auto small = [&](int i) {
            for (int c = 0; c < ncol; c++)
                if (std::fabs(h.arr[(size_t)(base + c) * n + i]) > thr) return false;
            return true;
        };
        for (int i = 0; i < n; i++)
            if (small(i)) { first = i; break; }
        if (first >= 0) {
            int last = first;
            while (last < n && small(last)) last++;
            h.corr_lo = first;
            h.corr_hi = last;
        }
    }
}

// Segment count and homogeneous responses for the segmented line solve.
// tri:   forward  x_n = -m_n x_{n-1}                        from x_{a-1} = 1
//        backward x_n = -c_n x_{n+1} rw_n                    from x_b = 1
// penta: forward  B_n = -m2_{n-1} B_{n-2} - m1_n B_{n-1}     from (B_{a-1}, B_{a-2}) = (1,0) | (0,1)
//        backward x_n = (-f_n x_{n+2} - C_n x_{n+1}) rD_n    from (x_b, x_{b+1}) = (1,0) | (0,1)
void segment(LineOpHost &h, int precision) {
    int n = h.N;
    bool tri = h.kind == K_TRI_PER || h.kind == K_TRI_DIR;
    bool pen = h.kind == K_PEN_PER || h.kind == K_PEN_DIR;
    h.S = 1;
    h.L = 0;
    if (!(tri || pen)) return;
    const int UB = 8;
    int S = 0;
    int Lr = reg_segment_len(n, h.kind, precision);
    if (Lr) {
        S = n / Lr;
        h.L = Lr;
    } else {
        for (int cand : {4, 2})
            if (n % cand == 0 && (n / cand) % UB == 0 && n / cand >= 32 && n / cand >= h.bw) { S = cand; break; }
    }
    if (!S) return;
    h.S = S;
    int L = n / S;
    auto A = [&](int a, int i) { return h.arr[(size_t)a * n + i]; };
    h.sfa.assign(n, 0.0);
    h.sfb.assign(n, 0.0);
    h.sba.assign(n, 0.0);
    h.sbb.assign(n, 0.0);
    for (int w = 0; w < S; w++) {
        int a = w * L, b = a + L;
        for (int which = 0; which < (pen ? 2 : 1); which++) {
            // forward
            double p1 = which == 0 ? 1.0 : 0.0, p2 = which == 0 ? 0.0 : 1.0;   // B_{n-1}, B_{n-2}
            for (int i = a; i < b; i++) {
                double x;
                if (tri) x = -A(0, i) * p1;
                else x = -(i >= 1 ? A(1, i - 1) : 0.0) * p2 - A(0, i) * p1;
                (which == 0 ? h.sfa : h.sfb)[i] = x;
                p2 = p1;
                p1 = x;
            }
            // backward
            double q1 = which == 0 ? 1.0 : 0.0, q2 = which == 0 ? 0.0 : 1.0;   // x_{n+1}, x_{n+2}
            for (int i = b - 1; i >= a; i--) {
                double x;
                if (tri) x = (0.0 - A(2, i) * q1) * A(1, i);
                else x = (0.0 - A(4, i) * q2 - A(3, i) * q1) * A(2, i);
                (which == 0 ? h.sba : h.sbb)[i] = x;
                q2 = q1;
                q1 = x;
            }
        }
    }
}

// Offsets (in elements) of the arrays inside one operator's device buffer.
struct Layout {
    size_t arr = 0, head = 0, tail = 0, seg = 0;
    size_t pf = 0, pb = 0, pz = 0, sf2 = 0, sb2 = 0, hp = 0, tp = 0, pbs = 0;
};

// Is the interior stencil of h antisymmetric with a zero centre (the first
// derivatives), so that a row's RHS is sum_k st[H+k] (phi[n+k] - phi[n-k])?
bool antisymmetric(const LineOpHost &h) {
    if (h.H < 1 || h.H > 3 || h.st[h.H] != 0.0) return false;
    for (int k = 1; k <= h.H; k++)
        if (h.st[h.H + k] != -h.st[h.H - k]) return false;
    for (int k = 2 * h.H + 1; k < 11; k++)
        if (h.st[k] != 0.0) return false;
    return true;
}

template <typename R>
void fill_dev(const LineOpHost &h, const char *base, const Layout &lo, LineOpDev<R> &d) {
    d.stat_lo = h.stat_lo;
    d.stat_hi = h.stat_hi;
    d.corr_lo = h.corr_lo;
    d.corr_hi = h.corr_hi;
    for (int i = 0; i < 5; i++) d.stat_c[i] = (R)h.stat_c[i];
    d.N = h.N;
    d.kind = h.kind;
    d.H = h.H;
    d.bw = h.bw;
    d.inv_dh = (R)h.inv_dh;
    for (int i = 0; i < 11; i++) d.st[i] = (R)h.st[i];
    for (int i = 0; i < 4; i++) d.sc[i] = (R)h.sc[i];
    for (int i = 0; i < 16; i++) d.Hm[i] = (R)h.Hm[i];
    for (int i = 0; i < 6; i++) d.cp[i] = (R)h.cp[i];
    d.asym = antisymmetric(h) ? 1 : 0;
    for (int k = 0; k < 3; k++) d.sta[k] = d.asym && k < h.H ? (R)(h.st[h.H + 1 + k] * h.inv_dh) : R(0);
    {
        // stationary backward factors: tri (c, rw) = stat_c[2], stat_c[1]; penta (C, f, rD) = stat_c[3], stat_c[4], stat_c[2]
        const bool tri = h.kind == K_TRI_PER || h.kind == K_TRI_DIR;
        const double C = tri ? h.stat_c[2] : h.stat_c[3], f = tri ? 0.0 : h.stat_c[4], rD = tri ? h.stat_c[1] : h.stat_c[2];
        d.stat_b[0] = (R)(C * rD);
        d.stat_b[1] = (R)(f * rD);
        d.stat_b[2] = (R)rD;
    }
    const R *p = (const R *)base;
    size_t n = h.N;
    size_t na = h.arr.size() / n;
    const R *a = p + lo.arr;
    d.a0 = na > 0 ? a : nullptr;
    d.a1 = na > 1 ? a + n : nullptr;
    d.a2 = na > 2 ? a + 2 * n : nullptr;
    d.a3 = na > 3 ? a + 3 * n : nullptr;
    d.a4 = na > 4 ? a + 4 * n : nullptr;
    d.z0 = na > 5 ? a + 5 * n : nullptr;
    d.z1 = na > 6 ? a + 6 * n : nullptr;
    d.z2 = na > 7 ? a + 7 * n : nullptr;
    d.z3 = na > 8 ? a + 8 * n : nullptr;
    d.head = h.head.empty() ? nullptr : p + lo.head;
    d.tail = h.tail.empty() ? nullptr : p + lo.tail;
    const R *sg = p + lo.seg;
    d.S = h.S;
    d.seg_kf = h.seg_kf;
    d.seg_kb = h.seg_kb;
    d.sfa = h.S > 1 ? sg : nullptr;
    d.sfb = h.S > 1 ? sg + n : nullptr;
    d.sba = h.S > 1 ? sg + 2 * n : nullptr;
    d.sbb = h.S > 1 ? sg + 3 * n : nullptr;
    d.L = h.L;
    d.pf = h.L ? p + lo.pf : nullptr;
    d.pb = h.L ? p + lo.pb : nullptr;
    d.pz = h.L && h.kind == K_PEN_PER ? p + lo.pz : nullptr;
    d.sf2 = h.L ? p + lo.sf2 : nullptr;
    d.sb2 = h.L ? p + lo.sb2 : nullptr;
    d.pbs = h.L ? p + lo.pbs : nullptr;
    const bool dir = h.kind == K_TRI_DIR || h.kind == K_PEN_DIR;
    d.hp = h.L && dir ? p + lo.hp : nullptr;
    d.tp = h.L && dir ? p + lo.tp : nullptr;
}

template <typename R>
std::vector<R> flatten(const LineOpHost &h, Layout &lo) {
    std::vector<R> v;
    auto put = [&](double x) { v.push_back((R)x); };
    auto align4 = [&]() {   // vector loads of 2 or 4 values need 16-byte aligned rows
        while (v.size() % 4) v.push_back((R)0);
    };
    lo.arr = v.size();
    for (double x : h.arr) put(x);
    lo.head = v.size();
    for (double x : h.head) put(x);
    lo.tail = v.size();
    for (double x : h.tail) put(x);
    lo.seg = v.size();
    if (h.S > 1)
        for (const std::vector<double> *a : {&h.sfa, &h.sfb, &h.sba, &h.sbb})
            for (double x : *a) put(x);
    if (h.L) {
        const int n = h.N;
        const bool tri = h.kind == K_TRI_PER || h.kind == K_TRI_DIR;
        auto A = [&](int a, int i) { return h.arr[(size_t)a * n + i]; };
        align4();
        lo.pf = v.size();
        for (int i = 0; i < n; i++) {
            put(i >= 1 ? A(0, i) : 0.0);
            put(!tri && i >= 2 ? A(1, i - 1) : 0.0);
        }
        align4();
        lo.pb = v.size();
        for (int i = 0; i < n; i++) {
            if (tri) {
                put(A(2, i));
                put(0.0);
                put(A(1, i));
            } else {
                put(A(3, i));
                put(A(4, i));
                put(A(2, i));
            }
            put(0.0);
        }
        align4();
        lo.pbs = v.size();
        for (int i = 0; i < n; i++) {
            const double C = tri ? A(2, i) : A(3, i), f = tri ? 0.0 : A(4, i), rD = tri ? A(1, i) : A(2, i);
            put(C * rD);
            put(f * rD);
            put(rD);
            put(0.0);
        }
        if (h.kind == K_PEN_PER) {
            align4();
            lo.pz = v.size();
            for (int i = 0; i < n; i++)
                for (int c = 0; c < 4; c++) put(A(5 + c, i));
        }
        align4();
        lo.sf2 = v.size();
        for (int i = 0; i < n; i++) {
            put(h.sfa[i]);
            put(h.sfb[i]);
        }
        align4();
        lo.sb2 = v.size();
        for (int i = 0; i < n; i++) {
            put(h.sba[i]);
            put(h.sbb[i]);
        }
        if (h.kind == K_TRI_DIR || h.kind == K_PEN_DIR) {
            const int bw = h.bw, B = MC3D_BWMAX;
            lo.hp = v.size();
            for (int r = 0; r < h.H; r++)
                for (int k = 0; k < B; k++) put(k < bw ? h.head[(size_t)r * bw + k] : 0.0);
            lo.tp = v.size();
            for (int r = 0; r < h.H; r++)
                for (int k = 0; k < B; k++) {
                    int kk = k - (B - bw);
                    put(kk >= 0 ? h.tail[(size_t)r * bw + kk] : 0.0);
                }
        }
    }
    if (v.empty()) v.push_back((R)0);
    return v;
}
}  // namespace

int reg_segment_len(int N, int kind, int precision) {
    if (!(kind == K_TRI_PER || kind == K_TRI_DIR || kind == K_PEN_PER || kind == K_PEN_DIR)) return 0;
    if (precision != MC3D_FP64 && N % 64 == 0 && N / 64 >= 2 && N / 64 <= 16) return 64;
    if (N % 32 == 0 && N / 32 >= 2 && N / 32 <= 16) return 32;
    return 0;
}

int upload_line_op(const LineOpHost &hin, int precision, LineOpBuf &out) {
    LineOpHost h = hin;
    if (h.bw > MC3D_BWMAX) return fail(MC3D_ERR_CONFIG, "boundary row wider than the kernels support");
    analyse(h, precision);
    segment(h, precision);
    if (h.S > 1) {
        // responses below 2^-64 (FP64) / 2^-32 (FP32) of their unit start are dropped
        const double thr = std::ldexp(1.0, precision == MC3D_FP64 ? -64 : -32);
        int n = h.N, L = n / h.S;
        h.seg_kf = h.seg_kb = 0;
        for (int w = 0; w < h.S; w++)
            for (int r = 0; r < L; r++) {
                int i = w * L + r;
                if (std::fabs(h.sfa[i]) > thr || std::fabs(h.sfb[i]) > thr) h.seg_kf = std::max(h.seg_kf, r + 1);
                if (std::fabs(h.sba[i]) > thr || std::fabs(h.sbb[i]) > thr) h.seg_kb = std::max(h.seg_kb, L - r);
            }
    }
    out.precision = precision;
    MC3D_CUDA_TRY(cudaGetDevice(&out.device));
    Layout lo;
    if (precision == MC3D_FP64) {
        std::vector<double> v = flatten<double>(h, lo);
        MC3D_CUDA_TRY(cudaMalloc(&out.dev, v.size() * sizeof(double)));
        MC3D_CUDA_TRY(cudaMemcpy(out.dev, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
        fill_dev<double>(h, (const char *)out.dev, lo, out.f64);
    } else {
        std::vector<float> v = flatten<float>(h, lo);
        MC3D_CUDA_TRY(cudaMalloc(&out.dev, v.size() * sizeof(float)));
        MC3D_CUDA_TRY(cudaMemcpy(out.dev, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice));
        fill_dev<float>(h, (const char *)out.dev, lo, out.f32);
    }
    return MC3D_OK;
}

void free_line_op(LineOpBuf &b) {
    if (b.dev) cudaFree(b.dev);
    b.dev = nullptr;
}

}  // namespace mc3d
