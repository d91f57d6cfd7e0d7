/* nvtx_record.c -- test-only NVTX tool that records range pushes and pops.
 *
 * The NVTX v3 header code inside liblesb200.so loads this library when the
 * process has NVTX_INJECTION64_PATH set to its build, and calls
 * InitializeInjectionNvtx2 once per module that uses NVTX.  Every
 * nvtxRangePushA appends "+<name>" and every nvtxRangePop appends "-" to the
 * file named by LES_NVTX_LOG, one line each. */
#define NVTX_NO_IMPL
#include <nvtx3/nvToolsExt.h>
#include <stdio.h>
#include <stdlib.h>

static FILE *g_log;

static int rec_push(const char *msg) {
    if (g_log) {
        fprintf(g_log, "+%s\n", msg ? msg : "");
        fflush(g_log);
    }
    return 0;
}

static int rec_pop(void) {
    if (g_log) {
        fputs("-\n", g_log);
        fflush(g_log);
    }
    return 0;
}

int InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get) {
    const char *path = getenv("LES_NVTX_LOG");
    if (!g_log && path) g_log = fopen(path, "a");
    if (!g_log || !get) return 0;
    const NvtxExportTableCallbacks *cb = (const NvtxExportTableCallbacks *)get(NVTX_ETID_CALLBACKS);
    NvtxFunctionTable t = 0;
    unsigned int n = 0;
    if (!cb || !cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE, &t, &n) || !t) return 0;
    if (n < NVTX_CBID_CORE_RangePop) return 0;
    *t[NVTX_CBID_CORE_RangePushA] = (NvtxFunctionPointer)rec_push;
    *t[NVTX_CBID_CORE_RangePop] = (NvtxFunctionPointer)rec_pop;
    return 1;
}
