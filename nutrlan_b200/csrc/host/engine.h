// Thick-restart Lanczos engine: device-resident basis, host FP64 control.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../../include/trlx.h"

namespace trlb {

struct Options {
    int basis_bits = 64;
    uint64_t seed = 0x243F6A8885A308D3ull;
    cudaStream_t stream = nullptr;
    int refine = -1;  // -1: default (on for 32-bit bases)
    int profile = 0;  // per-kernel-class CUDA-event timing
};

Options options_from(const trlx_options *o);

// Thread-local statistics of the last solve (trlx_get_last_stats).
trlx_stats &last_stats();

void run_trlan(trl_matvec op, trl_uo uo, trl_info *info, int nrow, int mev, double *eval,
               double *evec, int lde, int lwrk, double *wrk, const Options &opt);
void run_ztrlan(ztrl_matvec op, trl_info *info, int nrow, int mev, double *eval,
                trl_dcomplex *evec, int lde, trl_dcomplex *misc, int nmis, const Options &opt);

// Validation/clearing of info before a solve (reference trl_clear_counter,
// SRC/trlan.c:1217-1349).
void clear_counter(trl_info *info, int nrow, int mev, int lde);

bool is_device_pointer(const void *p);

// Per-process file name of the reference (trl_pe_filename,
// SRC/trlaux.c:1047): the prefix up to its first blank, then the rank
// zero-padded to the number of digits of npes.
std::string pe_filename(const char *prefix, int rank, int npes);

// The reference's diagnostic channel (trl_open_logfile / trl_reopen_logfile,
// SRC/trlaux.c:48-118): info->log_fp when the caller opened one, else the
// per-process file named by trl_set_debug's prefix, else stdout.  A file
// opened here is closed by the destructor.
struct LogOut {
    FILE *fp = stdout;
    bool own = false;
    explicit LogOut(trl_info *info, const char *mode = "a");
    ~LogOut();
    LogOut(const LogOut &) = delete;
    LogOut &operator=(const LogOut &) = delete;
};

// Frees the calling thread's cached device workspace.
void release_workspace();

}  // namespace trlb
