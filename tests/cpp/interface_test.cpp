// interface_test.cpp -- the C++ mirror of the SmaxKernels interface
// (include/smax_b200.hpp) used the way the reference's own tests use
// SMAX::Interface; every result is checked against plain host loops here.
//
//   interface_test            run all cases on the GPU, print PASS/FAIL lines
//   interface_test --no-gpu   expect register_kernel to fail cleanly (no device)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "smax_b200.hpp"

using namespace smax_b200;

namespace {

int failures = 0;

void report(const char *name, bool ok, double err) {
    std::printf("%s %s (err %.3e)\n", ok ? "PASS" : "FAIL", name, err);
    if (!ok) ++failures;
}

double rel_err(const std::vector<double> &a, const std::vector<double> &b) {
    double d = 0, r = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        d += (a[i] - b[i]) * (a[i] - b[i]);
        r += b[i] * b[i];
    }
    return r > 0 ? std::sqrt(d / r) : std::sqrt(d);
}

// 5-point Laplacian of an m x m grid (4 on the diagonal, -1 off it)
struct Crs {
    int n = 0;
    std::vector<int> rp, col;
    std::vector<double> val;
};

Crs laplace(int m) {
    Crs a;
    a.n = m * m;
    a.rp.push_back(0);
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
            const int r = i * m + j;
            auto add = [&](int c, double v) { a.col.push_back(c); a.val.push_back(v); };
            if (i > 0) add(r - m, -1);
            if (j > 0) add(r - 1, -1);
            add(r, 4);
            if (j + 1 < m) add(r + 1, -1);
            if (i + 1 < m) add(r + m, -1);
            a.rp.push_back((int)a.col.size());
        }
    return a;
}

Crs lower_of(const Crs &a) {
    Crs l;
    l.n = a.n;
    l.rp.push_back(0);
    for (int r = 0; r < a.n; ++r) {
        for (int j = a.rp[r]; j < a.rp[r + 1]; ++j)
            if (a.col[j] <= r) { l.col.push_back(a.col[j]); l.val.push_back(a.val[j]); }
        l.rp.push_back((int)l.col.size());
    }
    return l;
}

std::vector<double> host_spmv(const Crs &a, const std::vector<double> &x) {
    std::vector<double> y(a.n, 0.0);
    for (int r = 0; r < a.n; ++r)
        for (int j = a.rp[r]; j < a.rp[r + 1]; ++j) y[r] += a.val[j] * x[a.col[j]];
    return y;
}

}  // namespace

int main(int argc, char **argv) {
    const bool expect_no_gpu = argc > 1 && std::strcmp(argv[1], "--no-gpu") == 0;
    Interface smax;
    if (expect_no_gpu) {
        const int rc = smax.register_kernel("spmv", KernelType::SPMV, PlatformType::CUDA);
        bool threw = false;
        try {
            smax.kernel("spmv");
        } catch (const std::runtime_error &) {
            threw = true;
        }
        std::printf("%s no-device register_kernel=%d, kernel() threw=%d\n", rc == 1 && threw ? "PASS" : "FAIL", rc,
                    (int)threw);
        return rc == 1 && threw ? 0 : 1;
    }

    const Crs A = laplace(40);
    const int n = A.n;
    std::vector<double> x(n);
    for (int i = 0; i < n; ++i) x[i] = std::sin(0.37 * i) + 0.1;
    const std::vector<double> y_ref = host_spmv(A, x);

    // -- CRS SpMV, then swap_operands: y = A x, x' = A y
    {
        std::vector<double> y(n, 0.0), xx = x;
        smax.register_kernel("spmv", KernelType::SPMV, PlatformType::CUDA, IntType::INT32, FloatType::FLOAT64);
        Kernel *k = smax.kernel("spmv");
        k->register_A(A.n, A.n, (int)A.col.size(), A.col.data(), A.rp.data(), A.val.data());
        k->register_B(n, xx.data());
        k->register_C(n, y.data());
        const int rc = k->run();
        report("spmv_crs", rc == 0 && rel_err(y, y_ref) < 1e-12, rel_err(y, y_ref));
        k->swap_operands();
        k->run();
        const std::vector<double> y2 = host_spmv(A, y_ref);
        report("spmv_swap_operands", rel_err(xx, y2) < 1e-12, rel_err(xx, y2));
    }

    // -- SELL-C-sigma SpMV through Utils::convert_crs_to_scs (y in permuted order)
    {
        int nr, npad, nc, nch, ne, nz;
        int *cp, *cl, *cc, *perm;
        double *cv;
        smax.utils->convert_crs_to_scs<int, double, int>(A.n, A.n, (int)A.col.size(), A.col.data(), A.rp.data(),
                                                         A.val.data(), 8, 64, nr, npad, nc, nch, ne, nz, cp, cl,
                                                         cc, cv, perm);
        std::vector<double> xs(npad > n ? npad : n, 0.0), ys(npad > n ? npad : n, 0.0);
        for (int i = 0; i < n; ++i) xs[i] = x[i];
        smax.register_kernel("scs", KernelType::SPMV, PlatformType::CUDA);
        Kernel *k = smax.kernel("scs");
        k->set_mat_scs(true);
        k->register_A(8, 64, nr, npad, nc, nch, ne, nz, cp, cl, cc, cv, perm);
        k->register_B((int)xs.size(), xs.data());
        k->register_C((int)ys.size(), ys.data());
        const int rc = k->run();
        std::vector<double> y(n);
        for (int r = 0; r < n; ++r) y[r] = ys[perm[r]];
        report("spmv_scs", rc == 0 && rel_err(y, y_ref) < 1e-12, rel_err(y, y_ref));
        delete[] cp;
        delete[] cl;
        delete[] cc;
        delete[] cv;
        delete[] perm;
    }

    // -- row-major SpMM, 4 vectors
    {
        const int kv = 4;
        std::vector<double> X(n * kv), Y(n * kv, 0.0), Yr(n * kv, 0.0);
        for (int i = 0; i < n * kv; ++i) X[i] = std::cos(0.11 * i);
        for (int r = 0; r < n; ++r)
            for (int j = A.rp[r]; j < A.rp[r + 1]; ++j)
                for (int v = 0; v < kv; ++v) Yr[r * kv + v] += A.val[j] * X[A.col[j] * kv + v];
        smax.register_kernel("spmm", KernelType::SPMM, PlatformType::CUDA);
        Kernel *k = smax.kernel("spmm");
        k->set_vec_row_major(true);
        k->register_A(A.n, A.n, (int)A.col.size(), A.col.data(), A.rp.data(), A.val.data());
        k->register_B(n, kv, X.data());
        k->register_C(n, kv, Y.data());
        const int rc = k->run();
        report("spmm_row_major", rc == 0 && rel_err(Y, Yr) < 1e-12, rel_err(Y, Yr));
    }

    // -- SpGEMM C = A*A, checked through C x = A (A x)
    {
        ULL cn = 0, cm = 0, cz = 0;
        int *ccol = nullptr, *crp = nullptr;
        double *cval = nullptr;
        smax.register_kernel("spgemm", KernelType::SPGEMM, PlatformType::CUDA);
        Kernel *k = smax.kernel("spgemm");
        k->register_A(A.n, A.n, (int)A.col.size(), A.col.data(), A.rp.data(), A.val.data());
        k->register_B(A.n, A.n, (int)A.col.size(), A.col.data(), A.rp.data(), A.val.data());
        k->register_C(&cn, &cm, &cz, &ccol, &crp, &cval);
        const int rc = k->run();
        Crs C;
        C.n = (int)cn;
        C.rp.assign(crp, crp + cn + 1);
        C.col.assign(ccol, ccol + cz);
        C.val.assign(cval, cval + cz);
        const std::vector<double> cx = host_spmv(C, x), aax = host_spmv(A, y_ref);
        report("spgemm_AA", rc == 0 && cn == (ULL)n && rel_err(cx, aax) < 1e-12, rel_err(cx, aax));
        delete[] ccol;
        delete[] crp;
        delete[] cval;
    }

    // -- lower SpTRSV: x = L^-1 b (B = solution, C = right-hand side)
    {
        Crs L = lower_of(A);
        std::vector<double> xs(n, 0.0), b = y_ref, xr(n, 0.0);
        for (int r = 0; r < n; ++r) {
            double s = b[r], d = 1;
            for (int j = L.rp[r]; j < L.rp[r + 1]; ++j)
                if (L.col[j] == r) d = L.val[j];
                else s -= L.val[j] * xr[L.col[j]];
            xr[r] = s / d;
        }
        smax.register_kernel("sptrsv", KernelType::SPTRSV, PlatformType::CUDA);
        Kernel *k = smax.kernel("sptrsv");
        k->register_A(L.n, L.n, (int)L.col.size(), L.col.data(), L.rp.data(), L.val.data());
        k->register_B(n, xs.data());
        k->register_C(n, b.data());
        const int rc = k->run();
        report("sptrsv_lower", rc == 0 && rel_err(xs, xr) < 1e-12, rel_err(xs, xr));

        // level-scheduled flow: generate_perm -> apply_mat_perm -> set_mat_perm
        std::vector<int> perm(n), inv(n);
        smax.utils->generate_perm(n, A.rp.data(), A.col.data(), perm.data(), inv.data(), "RS");
        Crs P;
        P.n = n;
        P.rp.resize(n + 1);
        P.col.resize(A.col.size());
        P.val.resize(A.val.size());
        smax.utils->apply_mat_perm(n, const_cast<int *>(A.rp.data()), const_cast<int *>(A.col.data()),
                                   const_cast<double *>(A.val.data()), P.rp.data(), P.col.data(), P.val.data(),
                                   perm.data(), inv.data());
        Crs PL = lower_of(P);
        std::vector<double> bp(n), xp(n, 0.0), xpr(n, 0.0);
        smax.utils->apply_vec_perm(n, b.data(), bp.data(), perm.data());
        for (int r = 0; r < n; ++r) {
            double s = bp[r], d = 1;
            for (int j = PL.rp[r]; j < PL.rp[r + 1]; ++j)
                if (PL.col[j] == r) d = PL.val[j];
                else s -= PL.val[j] * xpr[PL.col[j]];
            xpr[r] = s / d;
        }
        smax.register_kernel("sptrsv_lvl", KernelType::SPTRSV, PlatformType::CUDA);
        Kernel *kl = smax.kernel("sptrsv_lvl");
        kl->set_mat_perm(true);
        kl->register_A(PL.n, PL.n, (int)PL.col.size(), PL.col.data(), PL.rp.data(), PL.val.data());
        kl->register_B(n, xp.data());
        kl->register_C(n, bp.data());
        const int rc2 = kl->run();
        report("sptrsv_level_scheduled", rc2 == 0 && smax.get_n_levels() > 0 && rel_err(xp, xpr) < 1e-12,
               rel_err(xp, xpr));
    }

    // -- the reference's error conventions
    {
        bool threw = false;
        try {
            smax.kernel("does_not_exist");
        } catch (const std::runtime_error &) {
            threw = true;
        }
        bool bad_count = false;
        try {
            smax.kernel("spmv")->register_A(1, 2, 3, 4);
        } catch (const std::runtime_error &) {
            bad_count = true;
        }
        const int cpu = smax.register_kernel("cpu", KernelType::SPMV, PlatformType::CPU);
        report("error_conventions", threw && bad_count && cpu == 1, 0.0);
    }

    // -- Jacobi solver on the Laplacian: the iteration count and solution of a
    //    host loop with the applications' rules (residual before the loop and
    //    every 5 iterations, measured on the first x_new buffer)
    {
        const Crs P = laplace(12);
        const int m = P.n;
        std::vector<double> b(m), D(m);
        for (int i = 0; i < m; ++i) b[i] = std::cos(0.21 * i);
        for (int r = 0; r < m; ++r)
            for (int j = P.rp[r]; j < P.rp[r + 1]; ++j)
                if (P.col[j] == r) D[r] = P.val[j];
        std::vector<double> x_old(m, 0.0), x_new(m, 0.0);
        std::vector<double> *xo = &x_old, *xn = &x_new, *first = &x_new;
        auto resid = [&]() {
            const std::vector<double> t = host_spmv(P, *first);
            double mx = 0.0;
            for (int i = 0; i < m; ++i) mx = std::fmax(mx, std::fabs(b[i] - t[i]));
            return mx;
        };
        double norm = resid();
        int it = 0;
        while (norm > 1e-8 && it < 1000) {
            const std::vector<double> s = host_spmv(P, *xo);
            for (int i = 0; i < m; ++i) (*xn)[i] = (b[i] - (s[i] - D[i] * (*xo)[i])) / D[i];
            std::swap(xo, xn);
            ++it;
            if (it % 5 == 0) norm = resid();
        }
        std::vector<double> x(m, 0.0);
        Solver s(Solver::JACOBI, (uint64_t)m, (uint64_t)P.col.size(), P.rp.data(), P.col.data(), P.val.data());
        const smax_solver_stats st = s.solve(b.data(), x.data());
        const double err = rel_err(x, *xo);
        report("jacobi_solver", st.n_iters == it && err < 1e-12 && (int)s.history().size() == st.n_checks, err);
    }
    return failures ? 1 : 0;
}
