// Internal definitions shared by the host translation units of
// libcmscan_gpu.so: the host copy of a configured model, its device plans,
// and the model handle behind the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cmscan_gpu.h"
#include "cm_internal.h"
#include "qdb_kernel.h"
#include "qdb_plan.h"
#include "sweep_plan.h"

namespace cmx {

void set_error(const std::string &msg);
struct HbDev;  // device tables of the HMM-banded scanner (hb_scan.cu)
void hb_free(HbDev *h);
struct TrqDev;  // device tables of the truncated QDB / non-banded scanner (trq_scan.cu)
void trq_free(TrqDev *t);
bool build_plan(const cmgpu_cm *cm, int semiring, int qdbidx, Plan &p);

// ---------------------------------------------------------------------------
// host copy of a configured CM
// ---------------------------------------------------------------------------
struct HostCM {
    cmgpu_cm view{};
    std::vector<int8_t> sttype, stid;
    std::vector<int32_t> cfirst, cnum, itsc, ioesc, iendsc, ibeginsc, dmin1, dmax1, dmin2, dmax2;
    std::vector<float> tsc, oesc, endsc, beginsc;

    bool load(const cmgpu_cm *c) {
        const int M = c->M;
        if (M < 2 || c->W < 1 || !c->sttype || !c->stid || !c->cfirst || !c->cnum || !c->tsc || !c->oesc ||
            !c->endsc || !c->beginsc || !c->itsc || !c->ioesc || !c->iendsc || !c->ibeginsc || !c->dmin1 ||
            !c->dmax1 || !c->dmin2 || !c->dmax2)
            return false;
        sttype.assign(c->sttype, c->sttype + M);
        stid.assign(c->stid, c->stid + M);
        cfirst.assign(c->cfirst, c->cfirst + M);
        cnum.assign(c->cnum, c->cnum + M);
        tsc.assign(c->tsc, c->tsc + (size_t)M * MAXC);
        oesc.assign(c->oesc, c->oesc + (size_t)M * ESC);
        endsc.assign(c->endsc, c->endsc + M);
        beginsc.assign(c->beginsc, c->beginsc + M);
        itsc.assign(c->itsc, c->itsc + (size_t)M * MAXC);
        ioesc.assign(c->ioesc, c->ioesc + (size_t)M * ESC);
        iendsc.assign(c->iendsc, c->iendsc + M);
        ibeginsc.assign(c->ibeginsc, c->ibeginsc + M);
        dmin1.assign(c->dmin1, c->dmin1 + M);
        dmax1.assign(c->dmax1, c->dmax1 + M);
        dmin2.assign(c->dmin2, c->dmin2 + M);
        dmax2.assign(c->dmax2, c->dmax2 + M);
        view = *c;
        view.sttype = sttype.data();
        view.stid = stid.data();
        view.cfirst = cfirst.data();
        view.cnum = cnum.data();
        view.tsc = tsc.data();
        view.oesc = oesc.data();
        view.endsc = endsc.data();
        view.beginsc = beginsc.data();
        view.itsc = itsc.data();
        view.ioesc = ioesc.data();
        view.iendsc = iendsc.data();
        view.ibeginsc = ibeginsc.data();
        view.dmin1 = dmin1.data();
        view.dmax1 = dmax1.data();
        view.dmin2 = dmin2.data();
        view.dmax2 = dmax2.data();
        // structural sanity: children inside [0, M), B children valid
        for (int v = 0; v < M; v++) {
            int st = sttype[v];
            if (st < 0 || st > 8) return false;
            if (st == E_ST) continue;
            if (st == B_ST) {
                if (cfirst[v] <= v || cfirst[v] >= M || cnum[v] <= v || cnum[v] >= M) return false;
                if (stid[cfirst[v]] != BEGL_S) return false;
            } else {
                if (cnum[v] < 1 || cnum[v] > MAXC || cfirst[v] < v || cfirst[v] + cnum[v] > M) return false;
                for (int yo = 0; yo < cnum[v]; yo++) {
                    int y = cfirst[v] + yo;
                    if (y == v && st != IL_ST && st != IR_ST) return false;
                }
            }
        }
        return true;
    }
};

struct DevPlan {
    Plan host;
    StateDev *states = nullptr;
    ChunkDev *chunks = nullptr;
    BeginDev *begins = nullptr;
    int32_t *level_start = nullptr, *wb = nullptr, *cb = nullptr, *init_off = nullptr;
    uint32_t *tsc = nullptr, *endsc = nullptr, *beginsc = nullptr, *esc = nullptr, *el_sca = nullptr,
             *esc_c = nullptr, *init_val = nullptr, *beginsc_all = nullptr;
    std::vector<double> cells_prefix, terms_prefix;  // per jrow, prefix over jrow = 1..W
    double cells_full = 0, terms_full = 0;
    // node-sweep kernel (sweep_scan.cu); sw_ok false when the model is outside its scope
    bool sw_ok = false;
    std::string sw_why;
    SweepPlan sw;
    SwState *sw_st = nullptr;
    uint8_t *sw_kid = nullptr;
    SwNode *sw_nodes = nullptr;
    SwIO *sw_io = nullptr;
    SwBif *sw_bifs = nullptr;
    uint32_t *init0 = nullptr;
    ~DevPlan() {
        cudaFree(sw_st);
        cudaFree(sw_kid);
        cudaFree(sw_nodes);
        cudaFree(sw_io);
        cudaFree(sw_bifs);
        cudaFree(init0);
        cudaFree(states);
        cudaFree(chunks);
        cudaFree(begins);
        cudaFree(level_start);
        cudaFree(wb);
        cudaFree(cb);
        cudaFree(init_off);
        cudaFree(tsc);
        cudaFree(endsc);
        cudaFree(beginsc);
        cudaFree(esc);
        cudaFree(el_sca);
        cudaFree(esc_c);
        cudaFree(init_val);
        cudaFree(beginsc_all);
    }
};

}  // namespace cmx

struct cmgpu_model {
    using DevPlan = cmx::DevPlan;
    using HostCM = cmx::HostCM;
    int device = 0;
    HostCM cm;
    std::mutex mu;
    std::map<int, std::unique_ptr<DevPlan>> plans;  // key semiring*8 + qdbidx
    uint16_t *ilog = nullptr;
    int ilog_nz = 0;
    std::vector<float> flog;  // host FLogsum table for null3
    cmx::HbDev *hb = nullptr;  // built on the first HMM-banded scan
    cmx::TrqDev *trq = nullptr;  // built on the first truncated QDB / non-banded scan
    // host-only scan plans of the allocation-free entry point (key semiring*8 + qdbidx)
    mutable std::mutex noalloc_mu;
    mutable std::map<int, std::unique_ptr<cmx::Plan>> noalloc_plans;
    ~cmgpu_model() {
        cudaFree(ilog);
        cmx::hb_free(hb);
        cmx::trq_free(trq);
    }
};


namespace cmx {
// score_correction_null3 (src/cp9.rs:6516-6528) with the model's null and omega
float null3_corr(const cmgpu_model *m, const float *comp, int len);
// Replays the reference's greedy report for one window from its reportable
// cells (sorted by j, d) and removes overlaps; appends to `out`.
void report_window(const cmgpu_model *m, int semiring, const Cand *c, size_t n, const uint8_t *frame,
                   int32_t i0, float cutoff, int do_null3, std::vector<cmgpu_hit> &out);
}  // namespace cmx
