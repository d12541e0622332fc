// The range-Doppler chain over CPIs of mixed shapes with one launch per stage
// (zkx_rd_worklist_*).  No counterpart in the reference: its Task1 pipeline runs one CPI
// per call (ZKX/Task1/pipeline/src/steps/step2/step2.cu:7-47, step3, step4).
//
// The items are grouped by plan.  Each group's compressed cubes and power planes sit
// contiguously in one library-owned allocation, so one bulk-copy tensor map per group
// covers all of its CPIs; per-CPI pointers (inputs, threshold and detection planes) live
// in device tables.  A stage runs as one work-list kernel over the groups it covers and
// as the plan's own kernels for the others, chosen so that every CPI gets the bits it
// gets alone (see the coverage rules in build_coverage).
#include <algorithm>
#include <climits>
#include <cstring>
#include <map>
#include <vector>

#include "tma.cuh"
#include "worklist.h"
#include "zkx_internal.h"

namespace zkx {
namespace {

struct WlGroup {
    zkx_rd_plan plan = nullptr;
    RdPlanView v{};
    int first = 0;              // position of the group's first item in the grouped order
    int count = 0;              // CPIs
    size_t compressed_off = 0;  // byte offsets into the scratch allocation
    size_t power_off = 0;
    int variant = 0;            // resolved compression kernel of one CPI alone
    bool comp_wl = false, dop_wl = false, cfar_wl = false;
};

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace
}  // namespace zkx

struct zkx_rd_worklist_s {
    std::vector<zkx_rd_work_item> items;  // grouped order
    std::vector<zkx::WlGroup> groups;
    char* scratch = nullptr;
    size_t scratch_bytes = 0;
    void** tables = nullptr;              // device: xs[count], thr[count], det[count]
    std::vector<zkx::WlCompressionParams> comp;
    std::vector<int> comp_ctas;
    std::vector<zkx::WlDopplerParams> dop;
    std::vector<int> dop_ctas;
    std::vector<zkx::WlCfarParams> cfar;
    std::vector<int> cfar_ctas;
    int cfar_geometry[4] = {0, 0, 0, 0};
    int launches = 0;
};

namespace zkx {
namespace {

void release(zkx_rd_worklist w)
{
    if (!w) return;
    cudaFree(w->scratch);
    cudaFree(w->tables);
    delete w;
}

float2* group_compressed(zkx_rd_worklist w, const WlGroup& g)
{
    return reinterpret_cast<float2*>(w->scratch + g.compressed_off);
}

float* group_power(zkx_rd_worklist w, const WlGroup& g)
{
    return reinterpret_cast<float*>(w->scratch + g.power_off);
}

// Which stages of a group the work-list kernels run.  The rules keep each CPI's bits
// equal to the CPI executed alone with its plan:
//   compression  a power-of-two range nfft of 64 .. 8192 whose plan runs the
//                one-launch-per-pulse-group transform or the persistent Stockham kernel
//                (the same bits) with the table's radix plan, not the four-step or cluster
//                kernels;
//   Doppler      a power-of-two Doppler nfft of 64 .. 1024 (the column count per CTA does
//                not change a result);
//   CFAR         accurate mode, the list's tiled window geometry, a tile choice with the
//                whole-tile sums (full or persistent) and a range nfft that is a multiple
//                of 4 (the plan's own launch then also takes the bulk-copy tile).
int build_coverage(zkx_rd_worklist w)
{
    bool have_geometry = false;
    for (WlGroup& g : w->groups) {
        const zkx_rd_desc& d = g.v.d;
        const int P = d.num_pulses, nr = g.v.range_nfft, nd = g.v.doppler_nfft;
        ZKX_TRY(resolve_compression_variant(P, nr, g.v.tuning.compression_variant, &g.variant));
        const int alt = compression_alt_radix(nr);
        g.comp_wl = wl_compression_length(nr) && (alt == 0 || g.v.tuning.compression_radix != alt) &&
                    (g.variant == ZKX_COMPRESSION_DEFAULT || g.variant == ZKX_COMPRESSION_PLAIN ||
                     g.variant == ZKX_COMPRESSION_PERSISTENT);
        g.dop_wl = wl_doppler_length(nd) && (nr & 1) == 0;
        uint32_t bw = 0, bh = 0;
        const int* gd = d.guard_cells;
        const int* rf = d.reference_cells;
        bool tiled = d.cfar_mode == ZKX_CFAR_ACCURATE && wl_cfar_geometry(gd[0], gd[1], rf[0], rf[1], &bw, &bh) &&
                     (nr & 3) == 0 &&
                     (g.v.tuning.cfar_tile == ZKX_CFAR_TILE_DEFAULT || g.v.tuning.cfar_tile == ZKX_CFAR_TILE_FULL ||
                      g.v.tuning.cfar_tile == ZKX_CFAR_TILE_STREAM);
        if (tiled && !have_geometry) {
            w->cfar_geometry[0] = gd[0];
            w->cfar_geometry[1] = gd[1];
            w->cfar_geometry[2] = rf[0];
            w->cfar_geometry[3] = rf[1];
            have_geometry = true;
        }
        g.cfar_wl = tiled && gd[0] == w->cfar_geometry[0] && gd[1] == w->cfar_geometry[1] &&
                    rf[0] == w->cfar_geometry[2] && rf[1] == w->cfar_geometry[3];
    }
    return ZKX_SUCCESS;
}

// The stage kernels' parameter blocks, kWlGroups groups per launch.
int build_params(zkx_rd_worklist w)
{
    const float2* const* xs = reinterpret_cast<const float2* const*>(w->tables);
    const int count = (int)w->items.size();
    float* const* thr = reinterpret_cast<float* const*>(w->tables + count);
    uint8_t* const* det = reinterpret_cast<uint8_t* const*>(w->tables + 2 * count);

    for (int cls : {0, 1})
    for (WlGroup& g : w->groups) {
        if (!g.comp_wl || wl_length_class(g.v.range_nfft) != cls) continue;
        const long long add = wl_compression_ctas(g.v.range_nfft, g.count * g.v.d.num_pulses);
        if (w->comp.empty() || w->comp.back().groups == kWlGroups || w->comp.back().cls != cls ||
            w->comp_ctas.back() + add > INT_MAX) {
            w->comp.emplace_back();
            std::memset(&w->comp.back(), 0, sizeof(WlCompressionParams));
            w->comp.back().cls = cls;
            w->comp_ctas.push_back(0);
        }
        WlCompressionParams& p = w->comp.back();
        WlCompressionGroup& e = p.g[p.groups++];
        e.xs = xs + g.first;
        e.spectrum = g.v.spectrum;
        e.y = group_compressed(w, g);
        e.pulses = g.v.d.num_pulses;
        e.samples = g.v.d.samples_per_pulse;
        e.nfft = g.v.range_nfft;
        e.rows = g.count * g.v.d.num_pulses;
        e.entry0 = w->comp_ctas.back();
        w->comp_ctas.back() += (int)add;
    }

    for (int cls : {0, 1})
    for (WlGroup& g : w->groups) {
        if (!g.dop_wl || wl_length_class(g.v.doppler_nfft) != cls) continue;
        const int nr = g.v.range_nfft, nd = g.v.doppler_nfft, P = g.v.d.num_pulses;
        const int C = wl_doppler_columns(nd);
        CUtensorMap map;
        if (!encode_tensor_map_2d_f32(&map, group_compressed(w, g), 2ull * nr, (uint64_t)g.count * P,
                                      (uint64_t)nr * sizeof(float2), 2 * C, wl_doppler_box_rows(nd))) {
            g.dop_wl = false;  // the plan's own Doppler launch instead
            continue;
        }
        const long long add = (long long)g.count * ((nr + C - 1) / C);
        if (add > INT_MAX) return fail(ZKX_INVALID_SHAPE, "rd_worklist_create: a plan's Doppler tiles exceed one launch");
        if (w->dop.empty() || w->dop.back().groups == kWlGroups || w->dop.back().cls != cls ||
            w->dop_ctas.back() + add > INT_MAX) {
            w->dop.emplace_back();
            std::memset(&w->dop.back(), 0, sizeof(WlDopplerParams));
            w->dop.back().cls = cls;
            w->dop_ctas.push_back(0);
        }
        WlDopplerParams& p = w->dop.back();
        WlDopplerGroup& e = p.g[p.groups++];
        e.map = map;
        e.window = g.v.doppler_window;
        e.power = group_power(w, g);
        e.pulses = P;
        e.nr = nr;
        e.nd = nd;
        e.tiles_x = (nr + C - 1) / C;
        e.entry0 = w->dop_ctas.back();
        w->dop_ctas.back() += (int)add;
    }

    for (WlGroup& g : w->groups) {
        if (!g.cfar_wl) continue;
        const int nr = g.v.range_nfft, nd = g.v.doppler_nfft;
        uint32_t bw = 0, bh = 0;
        wl_cfar_geometry(w->cfar_geometry[0], w->cfar_geometry[1], w->cfar_geometry[2], w->cfar_geometry[3], &bw,
                         &bh);
        CUtensorMap map;
        if (!encode_tensor_map_2d_f32(&map, group_power(w, g), (uint64_t)nr, (uint64_t)g.count * nd,
                                      (uint64_t)nr * sizeof(float), bw, bh)) {
            g.cfar_wl = false;
            continue;
        }
        const long long add = (long long)g.count * ((nr + 63) / 64) * ((nd + 63) / 64);
        if (add > INT_MAX) return fail(ZKX_INVALID_SHAPE, "rd_worklist_create: a plan's CFAR tiles exceed one launch");
        if (w->cfar.empty() || w->cfar.back().groups == kWlGroups || w->cfar_ctas.back() + add > INT_MAX) {
            w->cfar.emplace_back();
            std::memset(&w->cfar.back(), 0, sizeof(WlCfarParams));
            w->cfar_ctas.push_back(0);
        }
        WlCfarParams& p = w->cfar.back();
        WlCfarGroup& e = p.g[p.groups++];
        e.map = map;
        e.thr = thr + g.first;
        e.det = det + g.first;
        e.scale64 = g.v.alpha / (double)g.v.nref;
        e.scale32 = (float)e.scale64;
        e.rows = nd;
        e.cols = nr;
        e.tiles_x = (nr + 63) / 64;
        e.tiles_y = (nd + 63) / 64;
        e.entry0 = w->cfar_ctas.back();
        w->cfar_ctas.back() += (int)add;
    }

    // launch calls per run
    int n = (int)(w->comp.size() + w->dop.size() + w->cfar.size());
    for (const WlGroup& g : w->groups) {
        if (!g.comp_wl) n += (g.count + kMaxRowTable - 1) / kMaxRowTable;
        if (!g.dop_wl) n += 1;
        if (!g.cfar_wl) n += g.count;
    }
    for (const zkx_rd_work_item& it : w->items)
        if (it.power) ++n;
    w->launches = n;
    return ZKX_SUCCESS;
}

int launch_list(zkx_rd_worklist w, cudaStream_t s)
{
    // range compression
    for (size_t i = 0; i < w->comp.size(); ++i)
        ZKX_TRY(launch_compression_worklist(w->comp[i], w->comp_ctas[i], w->comp[i].cls, s));
    for (const WlGroup& g : w->groups) {
        if (g.comp_wl) continue;
        const zkx_rd_desc& d = g.v.d;
        for (int b0 = 0; b0 < g.count; b0 += kMaxRowTable) {
            const int cnt = std::min(kMaxRowTable, g.count - b0);
            const float2* table[kMaxRowTable];
            for (int b = 0; b < cnt; ++b) table[b] = static_cast<const float2*>(w->items[g.first + b0 + b].x);
            ZKX_TRY(launch_pulse_compression_table(table, cnt, d.num_pulses, d.samples_per_pulse, g.v.range_nfft,
                                                   g.v.spectrum,
                                                   group_compressed(w, g) + (size_t)b0 * d.num_pulses * g.v.range_nfft,
                                                   g.variant, s, g.v.tuning.compression_radix,
                                                   g.v.tuning.compression_ctas_per_sm));
        }
    }
    // Doppler + |.|^2
    for (size_t i = 0; i < w->dop.size(); ++i)
        ZKX_TRY(launch_doppler_worklist(w->dop[i], w->dop_ctas[i], w->dop[i].cls, s));
    for (const WlGroup& g : w->groups) {
        if (g.dop_wl) continue;
        ZKX_TRY(launch_pulse_doppler(group_compressed(w, g), g.v.d.num_pulses, g.v.range_nfft, g.v.doppler_nfft,
                                     g.v.doppler_window, nullptr, group_power(w, g), g.count,
                                     g.v.tuning.doppler_columns, s));
    }
    // CA-CFAR
    for (size_t i = 0; i < w->cfar.size(); ++i)
        ZKX_TRY(launch_cfar_worklist(w->cfar[i], w->cfar_ctas[i], w->cfar_geometry[0], w->cfar_geometry[1],
                                     w->cfar_geometry[2], w->cfar_geometry[3], s));
    for (const WlGroup& g : w->groups) {
        if (g.cfar_wl) continue;
        const zkx_rd_desc& d = g.v.d;
        const int nr = g.v.range_nfft, nd = g.v.doppler_nfft;
        const size_t map = (size_t)nd * nr;
        for (int b = 0; b < g.count; ++b) {
            const zkx_rd_work_item& it = w->items[g.first + b];
            const float* power = group_power(w, g) + b * map;
            if (d.cfar_mode == ZKX_CFAR_COMPAT)
                ZKX_TRY(launch_ca_cfar_compat(power, 2, nd, nr, d.guard_cells[0], d.guard_cells[1],
                                              d.reference_cells[0], d.reference_cells[1], (float)g.v.alpha, g.v.nref,
                                              g.v.cumulative, it.threshold, it.detections, s));
            else
                ZKX_TRY(launch_ca_cfar_accurate(power, nd, nr, d.guard_cells[0], d.guard_cells[1],
                                                d.reference_cells[0], d.reference_cells[1], g.v.alpha, g.v.nref,
                                                it.threshold, it.detections, 1, g.v.tuning.cfar_tile, s,
                                                g.v.tuning.cfar_ctas_per_sm));
        }
    }
    // power planes the caller asked for
    for (const WlGroup& g : w->groups) {
        const size_t map = (size_t)g.v.doppler_nfft * g.v.range_nfft;
        for (int b = 0; b < g.count; ++b) {
            float* dst = w->items[g.first + b].power;
            if (dst)
                ZKX_CUDA(cudaMemcpyAsync(dst, group_power(w, g) + b * map, map * sizeof(float),
                                         cudaMemcpyDeviceToDevice, s));
        }
    }
    return ZKX_SUCCESS;
}

}  // namespace
}  // namespace zkx

using namespace zkx;

extern "C" int zkx_rd_worklist_create(const zkx_rd_work_item* items, int count, zkx_rd_worklist* out)
{
    if (!items || !out) return fail(ZKX_INVALID_ARGUMENT, "rd_worklist_create: null pointer");
    *out = nullptr;
    if (count < 1 || count > 65535) return fail(ZKX_INVALID_SHAPE, "rd_worklist_create: count must be 1..65535");
    ZKX_TRY(ensure_device_ready());
    // group by plan, in order of first appearance, then longest range transforms first
    std::vector<WlGroup> groups;
    std::map<zkx_rd_plan, int> index;
    std::vector<std::vector<int>> members;
    for (int i = 0; i < count; ++i) {
        const zkx_rd_work_item& it = items[i];
        if (!it.plan || !it.x || !it.threshold || !it.detections)
            return fail(ZKX_INVALID_ARGUMENT, "rd_worklist_create: null plan, input or output");
        auto f = index.find(it.plan);
        if (f == index.end()) {
            WlGroup g;
            g.plan = it.plan;
            ZKX_TRY(rd_plan_view(it.plan, &g.v));
            if (g.v.d.precision != ZKX_PRECISION_FP32)
                return fail(ZKX_UNSUPPORTED_OPERATION, "rd_worklist_create: plans must have FP32 precision");
            f = index.emplace(it.plan, (int)groups.size()).first;
            groups.push_back(g);
            members.emplace_back();
        }
        members[f->second].push_back(i);
    }
    std::vector<int> order(groups.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return groups[a].v.range_nfft > groups[b].v.range_nfft; });

    auto* w = new zkx_rd_worklist_s;
    size_t off = 0;
    for (int gi : order) {
        WlGroup g = groups[gi];
        g.first = (int)w->items.size();
        g.count = (int)members[gi].size();
        for (int i : members[gi]) w->items.push_back(items[i]);
        const long long P = g.v.d.num_pulses, nr = g.v.range_nfft, nd = g.v.doppler_nfft;
        if (g.count * P > INT_MAX || g.count * nd > INT_MAX) {
            release(w);
            return fail(ZKX_INVALID_SHAPE, "rd_worklist_create: a plan's CPIs exceed kernel capacity");
        }
        g.compressed_off = off;
        off = align256(off + (size_t)g.count * P * nr * sizeof(float2));
        g.power_off = off;
        off = align256(off + (size_t)g.count * nd * nr * sizeof(float));
        w->groups.push_back(g);
    }
    w->scratch_bytes = off;
    cudaError_t e = cudaMalloc(&w->scratch, off);
    if (e == cudaSuccess) e = cudaMalloc(&w->tables, (size_t)3 * count * sizeof(void*));
    if (e != cudaSuccess) {
        release(w);
        return cuda_status(e, "rd_worklist_create allocation");
    }
    std::vector<void*> host((size_t)3 * count);
    for (int i = 0; i < count; ++i) {
        host[i] = const_cast<void*>(w->items[i].x);
        host[count + i] = w->items[i].threshold;
        host[2 * count + i] = w->items[i].detections;
    }
    e = cudaMemcpy(w->tables, host.data(), host.size() * sizeof(void*), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        release(w);
        return cuda_status(e, "rd_worklist_create table upload");
    }
    int rc = build_coverage(w);
    if (rc == ZKX_SUCCESS) rc = build_params(w);
    if (rc != ZKX_SUCCESS) {
        release(w);
        return rc;
    }
    *out = w;
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_worklist_launch(zkx_rd_worklist list, zkx_stream_t stream)
{
    if (!list) return fail(ZKX_INVALID_ARGUMENT, "rd_worklist_launch: null list");
    return launch_list(list, static_cast<cudaStream_t>(stream));
}

extern "C" int zkx_rd_worklist_info(zkx_rd_worklist list, int* launches, int* groups, long long* scratch_bytes)
{
    if (!list) return fail(ZKX_INVALID_ARGUMENT, "rd_worklist_info: null list");
    if (launches) *launches = list->launches;
    if (groups) *groups = (int)list->groups.size();
    if (scratch_bytes) *scratch_bytes = (long long)list->scratch_bytes;
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_worklist_destroy(zkx_rd_worklist list)
{
    release(list);
    return ZKX_SUCCESS;
}
