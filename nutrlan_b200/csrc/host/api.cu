// C entry points of libtrlan_b200.so: the reference's public API
// (INC/trlan.h, INC/ztrlan.h) plus the trlx_* extensions (include/trlx.h).
//
// Post-processing routines (trl_check_ritz, trl_rayleigh_quotients,
// trl_ritz_projection, ztrl_check_ritz) work where the caller's vectors
// live: device vectors with device kernels (the operator receives device
// pointers), host vectors with host loops (the operator is host code).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <memory>
#include <vector>

#include "../../../include/trlx.h"
#include "../kernels/lanczos_kernels.h"
#include "dense.h"
#include "engine.h"

using trlb::zd;

namespace {

// ---- small device helpers for the post-processing routines -----------------
template <class C>
__global__ void k_axpy(long n, double a, const C *x, C *y) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) y[i] = y[i] + a * x[i];
}
template <class C>
__global__ void k_scal(long n, double a, C *x) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] = a * x[i];
}
// In place V(:,0:k) <- V(:,0:k) * W (W k x k, column-major), one row per thread.
__global__ void k_row_gemm(long n, int k, double *V, long ldv, const double *W) {
    extern __shared__ double ws[];
    for (int i = threadIdx.x; i < k * k; i += blockDim.x) ws[i] = W[i];
    __syncthreads();
    const long stride = (long)gridDim.x * blockDim.x;
    double row[128];
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        for (int c = 0; c < k; ++c) row[c] = V[i + c * ldv];
        for (int j = 0; j < k; ++j) {
            double s = 0.0;
            for (int c = 0; c < k; ++c) s += row[c] * ws[c + j * k];
            V[i + j * ldv] = s;
        }
    }
}

struct DevScratch {
    trlb::Scratch s;
    double *d_out = nullptr;
    DevScratch() {
        s.max_blocks = 148 * 8;
        s.max_cols = 4;
        cudaMalloc(&s.partials, (size_t)s.max_blocks * 8 * sizeof(double));
        cudaMalloc(&s.tickets, sizeof(unsigned) * trlb::kNumTickets);
        cudaMemset(s.tickets, 0, sizeof(unsigned) * trlb::kNumTickets);
        cudaMalloc(&d_out, sizeof(double));
    }
    ~DevScratch() {
        cudaFree(s.partials);
        cudaFree(s.tickets);
        cudaFree(d_out);
    }
    double dot(const double *x, const double *y, long n) {
        trlb::launch_dot<double>(x, y, n, d_out, s, 0);
        double h = 0.0;
        cudaMemcpy(&h, d_out, sizeof(double), cudaMemcpyDeviceToHost);
        return h;
    }
    double dotz(const zd *x, const zd *y, long n) {
        trlb::launch_dot<zd>(x, y, n, d_out, s, 0);
        double h = 0.0;
        cudaMemcpy(&h, d_out, sizeof(double), cudaMemcpyDeviceToHost);
        return h;
    }
};

int nblk(long n) { return (int)std::max<long>(1, std::min<long>((n + 255) / 256, 148 * 8)); }

double host_dot(int n, const double *x, const double *y) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += x[i] * y[i];
    return s;
}

void print_check_table(trl_info *info, int ncol, const double *alpha, const double *beta, const double *eval,
                       const double *rq, const double *res, const double *err, int nrow, int *check) {
    trlb::LogOut log_out(info);
    FILE *fp = log_out.fp;
    if (info->stat != 0) *check = -4;
    std::fprintf(fp, "TRL_CHECK_RITZ: \n");
    std::fprintf(fp, "           Ritz value       res norm   res diff  est error  diff w rq  act. error\n");
    const double nn_tol = (double)nrow * nrow * info->tol;
    for (int i = 0; i < ncol; ++i) {
        if (beta && eval) {
            std::fprintf(fp, "%21.14f    %11.3e%11.3e%11.3e%11.3e %11.3e%11.3e\n", alpha[i], res[i], beta[i] - res[i],
                         err[i], rq[i] - alpha[i], eval[i] - alpha[i], eval[i]);
            if (std::fabs(beta[i] - res[i]) > 0.00001) --*check;
            if (std::fabs(rq[i] - alpha[i]) > nn_tol) --*check;
            if (std::fabs(eval[i] - alpha[i]) > 10 * nn_tol || std::fabs(eval[i] - alpha[i]) > 10 * err[i])
                --*check;
        } else if (beta) {
            std::fprintf(fp, "%21.14f    %11.3e%11.3e%11.3e%11.3e\n", alpha[i], res[i], beta[i] - res[i], err[i],
                         rq[i] - alpha[i]);
            if (std::fabs(beta[i] - res[i]) > 0.00001) --*check;
            if (std::fabs(rq[i] - alpha[i]) > nn_tol) --*check;
        } else if (eval) {
            std::fprintf(fp, "%21.14f     %11.3e           %11.3e%11.3e%11.3e%11.3e\n", alpha[i], res[i], err[i],
                         rq[i] - alpha[i], eval[i] - alpha[i], eval[i]);
        } else {
            std::fprintf(fp, "%21.14f    %11.5e           %11.3e%11.3e\n", alpha[i], res[i], err[i],
                         rq[i] - alpha[i]);
        }
    }
    if (info->nec < info->ned) *check = 1;
}

// Error estimates from residuals and the gaps between Ritz values
// (reference SRC/trlan.c:967-985).
void error_estimates(int ncol, const double *alpha, const double *res, double *err) {
    double gapl = alpha[ncol - 1] - alpha[0];
    for (int i = 0; i < ncol - 1; ++i) {
        double gapr = alpha[i + 1] - alpha[i];
        gapl = std::min(gapl, gapr);
        err[i] = res[i] >= gapl ? res[i] : res[i] * res[i] / gapl;
        gapl = gapr;
    }
    err[ncol - 1] = res[ncol - 1] >= gapl ? res[ncol - 1] : res[ncol - 1] * res[ncol - 1] / gapl;
}

// Cholesky (upper, A = R^T R) of an n x n column-major matrix; 0 on success.
int chol_upper(int n, double *A) {
    for (int j = 0; j < n; ++j) {
        double s = A[j + j * n];
        for (int k = 0; k < j; ++k) s -= A[k + j * n] * A[k + j * n];
        if (!(s > 0.0)) return j + 1;
        double r = std::sqrt(s);
        A[j + j * n] = r;
        for (int i = j + 1; i < n; ++i) {
            double t = A[j + i * n];
            for (int k = 0; k < j; ++k) t -= A[k + j * n] * A[k + i * n];
            A[j + i * n] = t / r;
        }
        for (int i = j + 1; i < n; ++i) A[i + j * n] = 0.0;
    }
    return 0;
}

}  // namespace

// ===========================================================================
extern "C" {

void trl_init_info(trl_info *info, int nrow, int mxlan, int lohi, int ned, double tol, int restart, int maxmv,
                   void *mpicomp) {
    // Defaults and normalisation of the reference (SRC/trl_comm_none.c:27-192).
    std::memset(info, 0, sizeof(*info));
    if (tol > 0) {
        info->tol = tol;
        if (info->tol <= DBL_MIN)
            info->tol = DBL_EPSILON;
        else if (info->tol > 1.0)
            info->tol = std::min(0.1, 1.0 / info->tol);
    } else {
        info->tol = std::sqrt(DBL_EPSILON);
    }
    info->restart = restart > 0 ? restart : 0;
    info->ntot = nrow;
    info->maxmv = maxmv > 0 ? maxmv : std::min(std::max(info->ntot, 1000), 1000 * ned);
    if (mpicomp != NULL) std::fprintf(stderr, "TRL_INIT_INFO:  ignoring MPI Comm.\n");
    info->mpicomp = NULL;
    info->maxlan = mxlan;
    if (mxlan <= ned) info->maxlan = ned + std::max(ned, 6);
    info->lohi = lohi;
    info->ned = ned;
    info->nloc = nrow;
    info->guess = 0;
    info->nec = 0;
    info->locked = 0;
    info->clk_rate = CLOCKS_PER_SEC;
    info->clk_max = (clock_t)9223372036854775807LL;
    info->tmv = -1;
    info->trgt = -DBL_MAX;
    info->tres = -1.0;
    info->crat = 1.0;
    info->my_pe = 0;
    info->npes = 1;
    info->log_io = 99;
    info->cpio = 98;
    // The reference leaves rfact unset here; a defined value keeps scheme 8
    // well-defined when trl_set_restart was not called.
    info->rfact = 0.0;
}

void trl_set_restart(trl_info *info, double rfact) { info->rfact = rfact; }

void trl_set_debug(trl_info *info, int msglvl, char *filename) {
    info->verbose = msglvl;
    if (filename != NULL) {
        std::strncpy(info->log_file, filename, sizeof(info->log_file) - 1);
        if (msglvl >= 0 && info->my_pe == 0)
            std::printf("TRLan will write diagnostic messages to files with prefix %s.\n", info->log_file);
    }
}

void trl_set_checkpoint(trl_info *info, int cpflag, char *file) {
    info->cpflag = cpflag;
    if (file != NULL) {
        std::strncpy(info->cpfile, file, sizeof(info->cpfile) - 1);
        if (info->verbose >= 0 && info->my_pe == 0)
            std::printf("TRLan will write checkpoint to files with prefix %s.\n", info->cpfile);
    }
}

void trl_set_iguess(trl_info *info, int nec, int iguess, int ncps, char *cpf) {
    (void)ncps;
    info->nec = nec;
    info->guess = iguess;
    if (cpf != NULL && cpf[0] != '\0') std::strncpy(info->oldcpf, cpf, sizeof(info->oldcpf) - 1);
    info->stat = 0;
    if (std::strlen(info->oldcpf) > 0 && info->guess > 1) {
        const std::string name = trlb::pe_filename(info->oldcpf, info->my_pe, info->npes);
        FILE *fp = std::fopen(name.c_str(), "r");
        if (fp)
            std::fclose(fp);
        else
            info->stat = -8;
    }
}

void trlan(trl_matvec op, trl_uo user_ortho, trl_info *info, int nrow, int mev, double *eval, double *evec, int lde,
           int lwrk, double *wrk) {
    trlb::run_trlan(op, user_ortho, info, nrow, mev, eval, evec, lde, lwrk, wrk, trlb::Options());
}

void trlx_trlan(trl_matvec op, trl_uo user_ortho, trl_info *info, int nrow, int mev, double *eval, double *evec,
                int lde, int lwrk, double *wrk, const trlx_options *opts) {
    trlb::run_trlan(op, user_ortho, info, nrow, mev, eval, evec, lde, lwrk, wrk, trlb::options_from(opts));
}

void ztrlan(ztrl_matvec op, trl_info *info, int nrow, int mev, double *eval, trl_dcomplex *evec, int lde,
            trl_dcomplex *misc, int nmis, double *dwrk, int ldwrk) {
    (void)dwrk;
    (void)ldwrk;
    trlb::run_ztrlan(op, info, nrow, mev, eval, evec, lde, misc, nmis, trlb::Options());
}

void trlx_ztrlan(ztrl_matvec op, trl_info *info, int nrow, int mev, double *eval, trl_dcomplex *evec, int lde,
                 trl_dcomplex *misc, int nmis, double *dwrk, int ldwrk, const trlx_options *opts) {
    (void)dwrk;
    (void)ldwrk;
    trlb::run_ztrlan(op, info, nrow, mev, eval, evec, lde, misc, nmis, trlb::options_from(opts));
}

void trlx_default_options(trlx_options *o) {
    if (!o) return;
    o->basis_bits = 64;
    o->seed = 0;
    o->stream = nullptr;
    o->refine = -1;
    o->profile = 0;
}

void trlx_get_last_stats(trlx_stats *s) {
    if (s) *s = trlb::last_stats();
}

void trlx_release_workspace(void) { trlb::release_workspace(); }

const char *trlx_version(void) { return "trlan-b200 0.1 (sm_100a)"; }

void trl_print_info(trl_info *info, int mvflop) {
    trlb::LogOut log_out(info);
    FILE *fp = log_out.fp;
    const double t_op = info->tick_o, t_tot = info->tick_t, t_res = info->tick_r, t_orth = info->tick_h;
    const double r_op = (t_op != 0 && mvflop > 0) ? (double)mvflop * info->matvec : 0.0;
    const double r_orth = info->rflp_h + info->flop_h;
    const double r_res = info->rflp_r + info->flop_r;
    const double r_tot = r_op > 0 ? (double)mvflop * info->matvec + info->rflp + info->flop : 0.0;
    std::fprintf(fp, "TRLAN execution summary (exit status =%d)\n", info->stat);
    const char *which = info->lohi > 0 ? "LARGEST" : (info->lohi < 0 ? "SMALLEST" : "EXTREME");
    std::fprintf(fp, "Number of %-8s eigenpairs     %10d (computed) %11d (wanted)\n", which, info->nec, info->ned);
    std::fprintf(fp, "Times the operator is applied:   %10d (MAX: %16d )\n", info->matvec, info->maxmv);
    std::fprintf(fp, "Problem size:                    %10d (PE: %4d) %11d (Global)\n", info->nloc, info->my_pe,
                 info->ntot);
    std::fprintf(fp, "Convergence tolerance:           %10.3e (rel) %16.3e (abs)\n", info->tol,
                 info->tol * info->anrm);
    std::fprintf(fp, "Maximum basis size:              %10d\n", info->maxlan);
    std::fprintf(fp, "Restarting scheme:               %10d\n", info->restart);
    std::fprintf(fp, "Number of re-orthogonalizations: %10d\n", info->north);
    std::fprintf(fp, "Number of (re)start loops:       %10d\n", info->nloop);
    if (info->nrand > 0) std::fprintf(fp, "Number of random vectors used:   %10d\n", info->nrand);
    std::fprintf(fp, "Number of eigenpairs locked:     %10d\n", info->locked);
    if (t_op > 0)
        std::fprintf(fp, "OP(MATVEC):            %12.4e sec, %12.4e FLOP/S (%11.4e FLOP)\n", t_op, r_op / t_op, r_op);
    else
        std::fprintf(fp, "time in OP:            %12.4e sec\n", t_op);
    if (t_orth > 0)
        std::fprintf(fp, "Re-Orthogonalization:: %12.4e sec, %12.4e FLOP/S (%11.4e FLOP)\n", t_orth, r_orth / t_orth,
                     r_orth);
    else
        std::fprintf(fp, "time in orth:          %12.4e sec\n", t_orth);
    if (t_res > 0)
        std::fprintf(fp, "Restarting::           %12.4e sec, %12.4e FLOP/S (%11.4e FLOP)\n", t_res, r_res / t_res, r_res);
    else
        std::fprintf(fp, "time in restarting:    %12.4e sec\n", t_res);
    if (t_tot > 0)
        std::fprintf(fp, "TRLAN on this PE:      %12.4e sec, %12.4e FLOP/S (%11.4e FLOP)\n", t_tot, r_tot / t_tot, r_tot);
    else
        std::fprintf(fp, "total time in TRLAN:   %12.4e sec\n", t_tot);
}

void trl_terse_info(trl_info *info, FILE *iou) {
    std::unique_ptr<trlb::LogOut> log_out;
    if (!iou) {
        log_out.reset(new trlb::LogOut(info));
        iou = log_out->fp;
    }
    const double t_op = info->tick_o, t_tot = info->tick_t, t_res = info->tick_r, t_orth = info->tick_h;
    const char sign = info->lohi > 0 ? '+' : (info->lohi < 0 ? '-' : '0');
    std::fprintf(iou, "MAXLAN:%10d, Restart:%10d,   NED: %c %7d,      NEC:%10d\n", info->maxlan, info->restart, sign,
                 info->ned, info->nec);
    std::fprintf(iou, "MATVEC:%10d,  Reorth:%10d, Nloop:   %7d,  Nlocked:%10d\n", info->matvec, info->north,
                 info->nloop, info->locked);
    if (t_tot > 0.001 && std::max(t_tot, std::max(t_op, std::max(t_res, t_orth))) < 1000)
        std::fprintf(iou, "Ttotal:%10.6f,    T_op:%10.6f, Torth:%10.6f,   Tstart:%10.6f\n", t_tot, t_op, t_orth, t_res);
    else
        std::fprintf(iou, "Ttotal:%10.3e,    T_op:%10.3e, Torth:%10.3e,   Tstart:%10.3e\n", t_tot, t_op, t_orth, t_res);
}

// Rayleigh quotient and residual norm of each Ritz pair (SRC/trlan.c:805).
void trl_check_ritz(trl_matvec op, trl_info *info, int nrow, int ncol, double *rvec, int ldrvec, double *alpha,
                    int *check, double *beta, double *eval, double *wrk, int lwrk) {
    (void)wrk;
    (void)lwrk;
    if (ncol <= 0) return;
    *check = 0;
    std::vector<double> rq(ncol), res(ncol), err(ncol);
    if (trlb::is_device_pointer(rvec)) {
        DevScratch ds;
        double *aq = nullptr;
        cudaMalloc(&aq, sizeof(double) * nrow);
        for (int i = 0; i < ncol; ++i) {
            const double *v = rvec + (long)i * ldrvec;
            op(nrow, 1, v, ldrvec, aq, nrow, info->mvparam);
            cudaDeviceSynchronize();
            rq[i] = ds.dot(v, aq, nrow);
            k_axpy<double><<<nblk(nrow), 256>>>(nrow, -rq[i], v, aq);
            res[i] = std::sqrt(ds.dot(aq, aq, nrow));
        }
        cudaFree(aq);
    } else {
        std::vector<double> aq(nrow);
        for (int i = 0; i < ncol; ++i) {
            const double *v = rvec + (long)i * ldrvec;
            op(nrow, 1, v, ldrvec, aq.data(), nrow, info->mvparam);
            rq[i] = host_dot(nrow, v, aq.data());
            for (int k = 0; k < nrow; ++k) aq[k] -= rq[i] * v[k];
            res[i] = std::sqrt(host_dot(nrow, aq.data(), aq.data()));
        }
    }
    error_estimates(ncol, alpha, res.data(), err.data());
    print_check_table(info, ncol, alpha, beta, eval, rq.data(), res.data(), err.data(), nrow, check);
}

void ztrl_check_ritz(ztrl_matvec op, trl_info *info, int nrow, int ncol, trl_dcomplex *rvec, int ldrvec,
                     double *alpha, int *check, double *beta, double *eval, trl_dcomplex *wrk, int lwrk) {
    (void)wrk;
    (void)lwrk;
    if (ncol <= 0) return;
    *check = 0;
    std::vector<double> rq(ncol), res(ncol), err(ncol);
    if (trlb::is_device_pointer(rvec)) {
        DevScratch ds;
        zd *aq = nullptr;
        cudaMalloc(&aq, sizeof(zd) * nrow);
        for (int i = 0; i < ncol; ++i) {
            const trl_dcomplex *v = rvec + (long)i * ldrvec;
            op(nrow, 1, v, ldrvec, reinterpret_cast<trl_dcomplex *>(aq), nrow, info->mvparam);
            cudaDeviceSynchronize();
            rq[i] = ds.dotz(reinterpret_cast<const zd *>(v), aq, nrow);
            k_axpy<zd><<<nblk(nrow), 256>>>(nrow, -rq[i], reinterpret_cast<const zd *>(v), aq);
            res[i] = std::sqrt(ds.dotz(aq, aq, nrow));
        }
        cudaFree(aq);
    } else {
        std::vector<trl_dcomplex> aq(nrow);
        for (int i = 0; i < ncol; ++i) {
            const trl_dcomplex *v = rvec + (long)i * ldrvec;
            op(nrow, 1, v, ldrvec, aq.data(), nrow, info->mvparam);
            double s = 0.0;
            for (int k = 0; k < nrow; ++k) s += v[k].r * aq[k].r + v[k].i * aq[k].i;
            rq[i] = s;
            double r2 = 0.0;
            for (int k = 0; k < nrow; ++k) {
                double xr = aq[k].r - s * v[k].r, xi = aq[k].i - s * v[k].i;
                r2 += xr * xr + xi * xi;
            }
            res[i] = std::sqrt(r2);
        }
    }
    error_estimates(ncol, alpha, res.data(), err.data());
    // The complex check floors the error estimate at machine epsilon times the
    // last Ritz value (SRC/ztrlan.c:393-397); the real check does not.
    for (int i = 0; i < ncol; ++i) err[i] = std::max(err[i], DBL_EPSILON * alpha[ncol - 1]);
    print_check_table(info, ncol, alpha, beta, eval, rq.data(), res.data(), err.data(), nrow, check);
}

// Normalise each vector, replace eres[i] by its Rayleigh quotient and
// eres[ncol+i] by its residual norm (SRC/trlan.c:1111-1215).
void trl_rayleigh_quotients(trl_matvec op, trl_info *info, int ncol, double *evec, int lde, double *eres,
                            double *base) {
    (void)base;
    const int nrow = info->nloc;
    if (ncol <= 0) return;
    if (info->verbose >= 0) {
        trlb::LogOut log_out(info);
    FILE *fp = log_out.fp;
        std::fprintf(fp, "TRLAN computing Rayleigh Quotients for %d Ritz pairs\n", ncol);
    }
    const bool dev = trlb::is_device_pointer(evec);
    DevScratch *ds = dev ? new DevScratch() : nullptr;
    double *aq = nullptr;
    std::vector<double> haq;
    if (dev)
        cudaMalloc(&aq, sizeof(double) * nrow);
    else
        haq.resize(nrow), aq = haq.data();
    for (int i = 0; i < ncol; ++i) {
        double *v = evec + (long)i * lde;
        double w0 = dev ? ds->dot(v, v, nrow) : host_dot(nrow, v, v);
        op(nrow, 1, v, lde, aq, nrow, info->mvparam);
        if (dev) cudaDeviceSynchronize();
        double w1 = dev ? ds->dot(v, aq, nrow) : host_dot(nrow, v, aq);
        info->matvec++;
        if (w0 > 0.0) {
            eres[i] = w1 / w0;
            if (dev)
                k_axpy<double><<<nblk(nrow), 256>>>(nrow, -eres[i], v, aq);
            else
                for (int k = 0; k < nrow; ++k) aq[k] -= eres[i] * v[k];
            double r2 = dev ? ds->dot(aq, aq, nrow) : host_dot(nrow, aq, aq);
            double inv = 1.0 / std::sqrt(w0);
            eres[ncol + i] = inv * std::sqrt(r2);
            if (dev)
                k_scal<double><<<nblk(nrow), 256>>>(nrow, inv, v);
            else
                for (int k = 0; k < nrow; ++k) v[k] *= inv;
        } else {
            eres[i] = -DBL_MAX;
            eres[ncol + i] = -DBL_MAX;
        }
    }
    if (dev) {
        cudaDeviceSynchronize();
        cudaFree(aq);
        delete ds;
    }
}

// Rayleigh-Ritz projection onto the first nev columns of evec
// (SRC/trlan.c:1438-1678): G = V'V = R'R, H = R^-T V'AV R^-1 = Y D Y',
// V <- V R^-1 Y, eres = (D, ||A v - d v||).  Unlike the reference, the
// residuals use A v - d v (the reference adds d v) and shifting for lohi > 0
// copies whole vectors.
void trl_ritz_projection(trl_matvec op, trl_info *info, int mev, double *evec, int lde, double *eres, double *wrk,
                         int lwrk, double *base) {
    (void)wrk;
    (void)lwrk;
    (void)base;
    const int nrow = info->nloc;
    int nev;
    if (info->nec > 0) {
        nev = info->nec + 1;
    } else {
        nev = std::min(info->ned, mev - 1);
        if (info->lohi != 0) nev++;
    }
    nev = std::min(nev, mev);
    if (info->verbose >= 0) {
        trlb::LogOut log_out(info);
    FILE *fp = log_out.fp;
        std::fprintf(fp, "TRLAN performing a Rayleigh-Ritz project for %d vectors.", nev);
    }
    if (nev <= 0 || nev > 128) {
        info->stat = -231;
        return;
    }
    const bool dev = trlb::is_device_pointer(evec);
    DevScratch *ds = dev ? new DevScratch() : nullptr;
    auto dot = [&](const double *x, const double *y) { return dev ? ds->dot(x, y, nrow) : host_dot(nrow, x, y); };
    std::vector<double> G((size_t)nev * nev), H((size_t)nev * nev);
    for (int j = 0; j < nev; ++j)
        for (int i = 0; i <= j; ++i) G[i + j * nev] = G[j + i * nev] = dot(evec + (long)i * lde, evec + (long)j * lde);
    if (chol_upper(nev, G.data())) {
        info->stat = -234;
        delete ds;
        return;
    }
    double *aq = nullptr;
    std::vector<double> haq;
    if (dev)
        cudaMalloc(&aq, sizeof(double) * nrow);
    else
        haq.resize(nrow), aq = haq.data();
    for (int j = 0; j < nev; ++j) {
        op(nrow, 1, evec + (long)j * lde, lde, aq, nrow, info->mvparam);
        if (dev) cudaDeviceSynchronize();
        for (int i = 0; i <= j; ++i) H[i + j * nev] = H[j + i * nev] = dot(evec + (long)i * lde, aq);
    }
    // H <- R^-T H R^-1 (R upper triangular in G).
    auto solve_rt = [&](std::vector<double> &M) {  // M <- R^-T M (forward substitution)
        for (int c = 0; c < nev; ++c)
            for (int i = 0; i < nev; ++i) {
                double s = M[i + c * nev];
                for (int k = 0; k < i; ++k) s -= G[k + i * nev] * M[k + c * nev];
                M[i + c * nev] = s / G[i + i * nev];
            }
    };
    solve_rt(H);
    std::vector<double> Ht((size_t)nev * nev);
    for (int i = 0; i < nev; ++i)
        for (int j = 0; j < nev; ++j) Ht[i + j * nev] = H[j + i * nev];
    solve_rt(Ht);
    std::vector<double> w(nev);
    if (trlb::sym_eig(nev, Ht.data(), nev, w.data())) {
        info->stat = -237;
        delete ds;
        return;
    }
    // Y <- R^-1 Y (back substitution).
    for (int c = 0; c < nev; ++c)
        for (int i = nev - 1; i >= 0; --i) {
            double s = Ht[i + c * nev];
            for (int k = i + 1; k < nev; ++k) s -= G[i + k * nev] * Ht[k + c * nev];
            Ht[i + c * nev] = s / G[i + i * nev];
        }
    if (dev) {
        double *dW = nullptr;
        cudaMalloc(&dW, sizeof(double) * nev * nev);
        cudaMemcpy(dW, Ht.data(), sizeof(double) * nev * nev, cudaMemcpyHostToDevice);
        k_row_gemm<<<nblk(nrow), 256, sizeof(double) * nev * nev>>>(nrow, nev, evec, lde, dW);
        cudaDeviceSynchronize();
        cudaFree(dW);
    } else {
        std::vector<double> row(nev);
        for (long i = 0; i < nrow; ++i) {
            for (int c = 0; c < nev; ++c) row[c] = evec[i + c * (long)lde];
            for (int j = 0; j < nev; ++j) {
                double s = 0.0;
                for (int c = 0; c < nev; ++c) s += row[c] * Ht[c + j * nev];
                evec[i + j * (long)lde] = s;
            }
        }
    }
    for (int i = 0; i < nev; ++i) {
        eres[i] = w[i];
        double *v = evec + (long)i * lde;
        op(nrow, 1, v, lde, aq, nrow, info->mvparam);
        if (dev) {
            cudaDeviceSynchronize();
            k_axpy<double><<<nblk(nrow), 256>>>(nrow, -w[i], v, aq);
        } else {
            for (int k = 0; k < nrow; ++k) aq[k] -= w[i] * v[k];
        }
        double r2 = dot(aq, aq);
        eres[nev + i] = r2 > 0.0 ? std::sqrt(r2) : -DBL_MAX;
    }
    if (info->lohi < 0) {
        for (int i = nev - 1; i < nev + nev - 2; ++i) eres[i] = eres[i + 1];
    } else if (info->lohi > 0) {
        for (int i = 0; i < nev - 1; ++i) {
            eres[i] = eres[i + 1];
            if (dev)
                cudaMemcpy(evec + (long)i * lde, evec + (long)(i + 1) * lde, sizeof(double) * nrow,
                           cudaMemcpyDeviceToDevice);
            else
                std::memcpy(evec + (long)i * lde, evec + (long)(i + 1) * lde, sizeof(double) * nrow);
        }
        for (int i = nev - 1; i < nev + nev - 2; ++i) eres[i] = eres[i + 2];
    }
    if (dev) {
        cudaFree(aq);
        delete ds;
    }
}

// ---- host building blocks ----------------------------------------------------
int trlx_host_get_eval(int nd, int locked, const double *alpha, const double *beta, double *lambda, double *res) {
    return trlb::get_eval(nd, locked, alpha, beta, lambda, res);
}
int trlx_host_tridiag_eig_last(int n, const double *d, const double *e, double *lambda, double *zlast) {
    return trlb::tridiag_eig_last(n, d, e, lambda, zlast);
}
int trlx_host_arrow_to_tridiag(int nd, const double *alpha, const double *beta, double *rot, double *alfrot,
                               double *betrot) {
    return trlb::arrow_to_tridiag(nd, alpha, beta, rot, alfrot, betrot);
}
int trlx_host_sym_eig(int n, double *A, int lda, double *w) { return trlb::sym_eig(n, A, lda, w); }
int trlx_host_herm_eig(int n, const trl_dcomplex *A, int lda, double *w, trl_dcomplex *Z, int ldz) {
    return trlb::herm_eig(n, reinterpret_cast<const std::complex<double> *>(A), lda, w,
                          reinterpret_cast<std::complex<double> *>(Z), ldz);
}
void trlx_host_shuffle_eig(int nd, int mnd, double *lambda, double *res, trl_info *info, int *kept, int locked) {
    trlb::shuffle_eig(nd, mnd, lambda, res, info, kept, locked);
}
void trlx_host_convergence_test(int nd, double *lambda, double *res, trl_info *info, double *wrk) {
    trlb::convergence_test(nd, lambda, res, info, wrk);
}
void trlx_host_sort_eig(int nd, int lohi, int nec, double ref, double *lambda, double *res) {
    trlb::sort_eig(nd, lohi, nec, ref, lambda, res);
}
void trlx_host_set_locking(int jnd, int nlam, double *lambda, double *res, double *yy, double anrm, int *locked) {
    trlb::set_locking(jnd, nlam, lambda, res, yy, anrm, locked);
}
void trlx_host_sort2(int n, double *key, double *other) { trlb::sort2(n, key, other); }

}  // extern "C"
