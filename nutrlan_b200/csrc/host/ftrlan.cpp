// Fortran-callable entry points (include/ftrlan.h).  Scalars arrive by
// reference; CHARACTER arguments are blank-padded with explicit lengths;
// the operator has no mvparam, so a per-thread trampoline adapts it to the
// C operator type the solver calls.
#include <cstring>
#include <string>

#include "../../../include/ftrlan.h"

namespace {

thread_local trl_fmatvec g_fop = nullptr;
thread_local ztrl_fmatvec g_zfop = nullptr;

void real_trampoline(const int nrow, const int ncol, const double *x, const int ldx, double *y, const int ldy,
                     void *) {
    int n = nrow, c = ncol, lx = ldx, ly = ldy;
    g_fop(&n, &c, const_cast<double *>(x), &lx, y, &ly);
}

void cplx_trampoline(const int nrow, const int ncol, const trl_dcomplex *x, const int ldx, trl_dcomplex *y,
                     const int ldy, void *) {
    int n = nrow, c = ncol, lx = ldx, ly = ldy;
    g_zfop(&n, &c, const_cast<trl_dcomplex *>(x), &lx, y, &ly);
}

// Fortran CHARACTER (blank-padded, not terminated) -> C string.
std::string fstring(const char *s, size_t len) {
    if (!s) return std::string();
    size_t n = 0;
    while (n < len && s[n] != '\0') ++n;
    while (n > 0 && s[n - 1] == ' ') --n;
    return std::string(s, n);
}

}  // namespace

extern "C" {

void trlan_(trl_fmatvec op, trl_info *info, int *nrow, int *mev, double *eval, double *evec, int *lde, int *lwrk,
            double *wrk) {
    trl_fmatvec saved = g_fop;
    g_fop = op;
    trlan(real_trampoline, nullptr, info, *nrow, *mev, eval, evec, *lde, *lwrk, wrk);
    g_fop = saved;
}

void ztrlan_(ztrl_fmatvec op, trl_info *info, int *nrow, int *mev, double *eval, trl_dcomplex *evec, int *lde,
             trl_dcomplex *misc, int *nmis, double *dwrk, int *ldwrk) {
    ztrl_fmatvec saved = g_zfop;
    g_zfop = op;
    ztrlan(cplx_trampoline, info, *nrow, *mev, eval, evec, *lde, misc, *nmis, dwrk, *ldwrk);
    g_zfop = saved;
}

void trl_init_info_(trl_info *info, int *nrow, int *mxlan, int *lohi, int *ned, double *tol, int *restart,
                    int *maxmv) {
    trl_init_info(info, *nrow, *mxlan, *lohi, *ned, *tol, *restart, *maxmv, nullptr);
}

void trl_set_restart_(trl_info *info, double *rfact) { trl_set_restart(info, *rfact); }

void trl_set_debug_(trl_info *info, int *msglvl, char *filename, size_t filename_len) {
    std::string f = fstring(filename, filename_len);
    trl_set_debug(info, *msglvl, f.empty() ? nullptr : &f[0]);
}

void trl_set_iguess_(trl_info *info, int *nec, int *iguess, int *nopts, char *cpf, size_t cpf_len) {
    std::string f = fstring(cpf, cpf_len);
    trl_set_iguess(info, *nec, *iguess, *nopts, f.empty() ? nullptr : &f[0]);
}

void trl_set_checkpoint_(trl_info *info, int *cpflag, char *file, size_t file_len) {
    std::string f = fstring(file, file_len);
    trl_set_checkpoint(info, *cpflag, f.empty() ? nullptr : &f[0]);
}

void trl_print_info_(trl_info *info, int *mvflop) { trl_print_info(info, *mvflop); }

}  // extern "C"
