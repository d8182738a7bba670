// A level split over several processes: halo exchange tables and the step
// taken one sweep at a time, so a host driver can exchange the ghost slabs
// of boxes owned by other ranks between sweeps (the FillBoundary of
// bamrexBCData::fill_consv_boundary across ranks, called after every sweep
// at Source/AmrLevelAdv_advance.cpp:356).  The level holds only this rank's
// boxes; its own ghost fill covers copies between them and the physical
// boundaries, and the host driver supplies the rest through these buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "bamrex_cuda.h"
#include "level_impl.h"

using namespace bamrex;

extern "C" int bamrex_level_set_halo(bamrex_level* L, int dir, const bamrex_region* send, int nsend,
                                     const bamrex_region* recv, int nrecv)
{
    if (!L || dir < 0 || dir >= L->D || nsend < 0 || nrecv < 0 || (nsend && !send) || (nrecv && !recv))
        return fail(BAMREX_ERR_ARG, "bad argument");
    const int nb = (int)L->boxes.size();
    std::vector<PackBox> pb[2];
    std::vector<FabDev> fb[2][2];
    const bamrex_region* src[2] = { send, recv };
    const int cnt[2] = { nsend, nrecv };
    long long cells[2] = { 0, 0 };
    for (int s = 0; s < 2; ++s) {
        for (int q = 0; q < cnt[s]; ++q) {
            const bamrex_region& r = src[s][q];
            if (r.box < 0 || r.box >= nb) return L->set_err(fail(BAMREX_ERR_ARG, "halo region names an unknown box"));
            const bamrex_box& B = L->boxes[r.box];
            for (int d = 0; d < 3; ++d) {
                const int g = d < L->D ? L->ngrow : 0;
                if (r.hi[d] < r.lo[d] || r.lo[d] < B.lo[d] - g || r.hi[d] > B.hi[d] + g)
                    return L->set_err(fail(BAMREX_ERR_ARG, "halo region outside its box's fab"));
            }
            if (r.offset != cells[s]) return L->set_err(fail(BAMREX_ERR_ARG, "halo regions must be packed in order"));
            PackBox p;
            for (int d = 0; d < 3; ++d) {
                p.lo[d] = r.lo[d];
                p.hi[d] = r.hi[d];
            }
            p.cell_begin = r.offset;
            cells[s] += (long long)(r.hi[0] - r.lo[0] + 1) * (r.hi[1] - r.lo[1] + 1) * (r.hi[2] - r.lo[2] + 1);
            pb[s].push_back(p);
            for (int par = 0; par < 2; ++par) fb[s][par].push_back(L->fab[par][r.box]);
        }
    }
    if (L->halo_mem[dir]) {
        cudaStreamSynchronize(L->stream);
        dev_free(L->halo_mem[dir], L->stream);
        L->halo_mem[dir] = nullptr;
    }
    size_t off = 0;
    size_t o_pb[2], o_fb[2][2];
    for (int s = 0; s < 2; ++s) {
        o_pb[s] = off;
        off = align_up(off + sizeof(PackBox) * std::max<size_t>(1, pb[s].size()), 256);
        for (int par = 0; par < 2; ++par) {
            o_fb[s][par] = off;
            off = align_up(off + sizeof(FabDev) * std::max<size_t>(1, fb[s][par].size()), 256);
        }
    }
    cudaError_t e = dev_alloc((void**)&L->halo_mem[dir], off, L->stream);
    if (e != cudaSuccess) return L->set_err(fail(BAMREX_ERR_OOM, "allocation of the halo tables failed"));
    char* m = L->halo_mem[dir];
    bamrex_level::Halo* H[2] = { &L->halo_send[dir], &L->halo_recv[dir] };
    for (int s = 0; s < 2; ++s) {
        H[s]->boxes = (PackBox*)(m + o_pb[s]);
        H[s]->nops = (int)pb[s].size();
        H[s]->cells = cells[s];
        if (!pb[s].empty())
            e = cudaMemcpyAsync(H[s]->boxes, pb[s].data(), sizeof(PackBox) * pb[s].size(), cudaMemcpyHostToDevice, L->stream);
        for (int par = 0; par < 2 && e == cudaSuccess; ++par) {
            H[s]->fabs[par] = (FabDev*)(m + o_fb[s][par]);
            if (!fb[s][par].empty())
                e = cudaMemcpyAsync(H[s]->fabs[par], fb[s][par].data(), sizeof(FabDev) * fb[s][par].size(),
                                    cudaMemcpyHostToDevice, L->stream);
        }
        if (e != cudaSuccess) return L->set_err(cuda_fail(e, "halo table upload"));
    }
    return BAMREX_OK;
}

extern "C" int bamrex_level_halo_pack(bamrex_level* L, int dir, double* sendbuf)
{
    if (!L || dir < 0 || dir >= L->D) return fail(BAMREX_ERR_ARG, "bad argument");
    const auto& h = L->halo_send[dir];
    if (!h.cells) return BAMREX_OK;
    if (!sendbuf) return L->set_err(fail(BAMREX_ERR_ARG, "NULL buffer"));
    return level_launch(L, launch_pack(L->NC, L->fp32, h.fabs[L->cur], h.boxes, h.nops, h.cells, sendbuf, 1, L->stream),
                        "halo pack");
}

extern "C" int bamrex_level_halo_unpack(bamrex_level* L, int dir, const double* recvbuf)
{
    if (!L || dir < 0 || dir >= L->D) return fail(BAMREX_ERR_ARG, "bad argument");
    const auto& h = L->halo_recv[dir];
    if (!h.cells) return BAMREX_OK;
    if (!recvbuf) return L->set_err(fail(BAMREX_ERR_ARG, "NULL buffer"));
    return level_launch(L, launch_pack(L->NC, L->fp32, h.fabs[L->cur], h.boxes, h.nops, h.cells, const_cast<double*>(recvbuf),
                                       0, L->stream),
                        "halo unpack");
}

extern "C" int bamrex_level_fill_dir(bamrex_level* L, int dir)
{
    if (!L || dir < 0 || dir >= L->D) return fail(BAMREX_ERR_ARG, "bad argument");
    return level_fill(L, dir, L->cur, nullptr);
}

extern "C" int bamrex_level_sweep_dir(bamrex_level* L, int dir, double dt, int reduce_ws)
{
    if (!L || dir < 0 || dir >= L->D) return fail(BAMREX_ERR_ARG, "bad argument");
    if (!(dt > 0)) return L->set_err(fail(BAMREX_ERR_ARG, "dt must be positive"));
    if (!L->reg_tasks[dir].empty())
        return L->set_err(fail(BAMREX_ERR_UNSUPPORTED, "flux registers are recorded by bamrex_level_advance only"));
    if (reduce_ws) {
        const cudaError_t e = cudaMemsetAsync(&L->d_scal->ws_bits, 0, sizeof(unsigned long long), L->stream);
        if (e != cudaSuccess) return L->set_err(cuda_fail(e, "memset"));
    }
    BX_TRY(level_sweep(L, dir, L->cur, dt, nullptr, reduce_ws != 0, true));
    L->cur ^= 1;
    L->ws_valid = reduce_ws != 0;
    return BAMREX_OK;
}

extern "C" int bamrex_level_wave_speed(bamrex_level* L, double* ws)
{
    if (!L || !ws) return fail(BAMREX_ERR_ARG, "NULL argument");
    if (!L->ws_valid) {
        cudaError_t e = cudaMemsetAsync(&L->d_scal->ws_bits, 0, sizeof(unsigned long long), L->stream);
        if (e != cudaSuccess) return L->set_err(cuda_fail(e, "memset"));
        BX_TRY(level_launch(L, launch_max_wave_speed(L->D, L->fp32, L->d_fab[L->cur], L->d_pack, (int)L->boxes.size(),
                                                     L->ncells, L->k, &L->d_scal->ws_bits, nullptr, L->stream),
                            "max wave speed"));
    }
    unsigned long long bits = 0;
    cudaError_t e = cudaMemcpyAsync(&bits, &L->d_scal->ws_bits, sizeof(bits), cudaMemcpyDeviceToHost, L->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "wave speed"));
    L->ws_valid = true;
    std::memcpy(ws, &bits, sizeof(double));
    return BAMREX_OK;
}

// ---------------------------------------------------------------------------
// The split step with its time step on the device.  Per step a host driver
// enqueues, without waiting: the halo exchange and sweep of each direction
// (dt read from the level's step scalars), a copy of this rank's max wave
// speed into a device buffer, an all-reduce MAX of that buffer over the
// ranks (NCCL on the level's stream), and bamrex_level_dist_dt, which
// takes the global max and sets the next dt (estTimeStep and the stop-time
// clamp of computeNewDt, Source/AmrLevelAdv.cpp:395-477, 600-611).

extern "C" int bamrex_level_dist_begin(bamrex_level* L, double time, double stop_time)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    if (L->run_pending) return L->set_err(fail(BAMREX_ERR_ARG, "a run is pending: call bamrex_level_run_wait"));
    StepScalars* h = L->h_scal;
    std::memset(h, 0, sizeof(*h));
    h->time = time;
    h->stop_time = stop_time;
    cudaError_t e = cudaMemcpyAsync(L->d_scal, h, sizeof(StepScalars), cudaMemcpyHostToDevice, L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "scalars upload"));
    BX_TRY(level_launch(L, launch_max_wave_speed(L->D, L->fp32, L->d_fab[L->cur], L->d_pack, (int)L->boxes.size(),
                                                 L->ncells, L->k, &L->d_scal->ws_bits, L->d_scal, L->stream),
                        "max wave speed"));
    L->run_pending = true;
    L->run_start_parity = L->cur;
    return BAMREX_OK;
}

extern "C" int bamrex_level_wave_speed_async(bamrex_level* L, double* dst_device)
{
    if (!L || !dst_device) return fail(BAMREX_ERR_ARG, "NULL argument");
    if (!L->run_pending) return L->set_err(fail(BAMREX_ERR_ARG, "call bamrex_level_dist_begin first"));
    // a max of non-negative doubles kept as their bit patterns: the bits are
    // the double
    const cudaError_t e = cudaMemcpyAsync(dst_device, &L->d_scal->ws_bits, sizeof(double), cudaMemcpyDeviceToDevice, L->stream);
    return e == cudaSuccess ? BAMREX_OK : L->set_err(cuda_fail(e, "wave speed copy"));
}

extern "C" int bamrex_level_dist_dt(bamrex_level* L, const double* ws_device, int first)
{
    if (!L || !ws_device) return fail(BAMREX_ERR_ARG, "NULL argument");
    if (!L->run_pending) return L->set_err(fail(BAMREX_ERR_ARG, "call bamrex_level_dist_begin first"));
    const cudaError_t e = cudaMemcpyAsync(&L->d_scal->ws_bits, ws_device, sizeof(double), cudaMemcpyDeviceToDevice, L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "wave speed copy"));
    return level_launch(L, launch_step_dt(L->d_scal, L->D, L->dx[0], L->dx[1], L->dx[2], L->cfl, first ? 0 : 1, L->stream),
                        "step dt");
}

extern "C" int bamrex_level_fill_dir_device(bamrex_level* L, int dir)
{
    if (!L || dir < 0 || dir >= L->D) return fail(BAMREX_ERR_ARG, "bad argument");
    if (!L->run_pending) return L->set_err(fail(BAMREX_ERR_ARG, "call bamrex_level_dist_begin first"));
    return level_fill(L, dir, L->cur, L->d_scal);
}

extern "C" int bamrex_level_sweep_dir_device(bamrex_level* L, int dir, int reduce_ws)
{
    if (!L || dir < 0 || dir >= L->D) return fail(BAMREX_ERR_ARG, "bad argument");
    if (!L->run_pending) return L->set_err(fail(BAMREX_ERR_ARG, "call bamrex_level_dist_begin first"));
    if (!L->reg_tasks[dir].empty())
        return L->set_err(fail(BAMREX_ERR_UNSUPPORTED, "flux registers are recorded by bamrex_level_advance only"));
    // the step scalars' ws_bits is zero here: bamrex_level_dist_dt cleared it
    BX_TRY(level_sweep(L, dir, L->cur, 0.0, L->d_scal, reduce_ws != 0, true));
    L->cur ^= 1;
    return BAMREX_OK;
}

extern "C" int bamrex_level_set_sweep_split(bamrex_level* L, int dir, const int* boxes, int nboxes)
{
    if (!L || dir < 0 || dir >= L->D || nboxes < 0 || (nboxes > 0 && !boxes)) return fail(BAMREX_ERR_ARG, "bad argument");
    const int nb = (int)L->boxes.size();
    std::vector<char> in_part1((size_t)nb, 0);
    for (int i = 0; i < nboxes; ++i) {
        if (boxes[i] < 0 || boxes[i] >= nb) return L->set_err(fail(BAMREX_ERR_ARG, "split box index out of range"));
        in_part1[(size_t)boxes[i]] = 1;
    }
    // the level's own tables, each box entry kept as it is (kernel shape,
    // tensor map, segments) and renumbered within its part
    std::vector<SweepBox> full[2];
    cudaError_t e = cudaSuccess;
    for (int p = 0; p < 2 && e == cudaSuccess; ++p) {
        full[p].resize((size_t)nb);
        e = cudaMemcpyAsync(full[p].data(), L->d_sweep[dir][p], sizeof(SweepBox) * nb, cudaMemcpyDeviceToHost, L->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "sweep split tables"));
    std::vector<SweepBox> part[2][2];  // [parity][part]
    long long items[2] = { 0, 0 };
    for (int b = 0; b < nb; ++b) {
        const int q = in_part1[(size_t)b];
        const long long n = (b + 1 < nb ? full[0][(size_t)b + 1].item_begin : L->items[dir]) - full[0][(size_t)b].item_begin;
        for (int p = 0; p < 2; ++p) {
            SweepBox sb = full[p][(size_t)b];
            sb.item_begin = items[q];
            part[p][q].push_back(sb);
        }
        items[q] += n;
    }
    dev_free(L->split_mem[dir], L->stream);
    L->split_mem[dir] = nullptr;
    char* mem = nullptr;
    e = dev_alloc((void**)&mem, sizeof(SweepBox) * (size_t)std::max(1, 2 * nb), L->stream);
    if (e != cudaSuccess) return L->set_err(fail(BAMREX_ERR_OOM, "sweep split tables"));
    L->split_mem[dir] = mem;
    size_t off = 0;
    for (int p = 0; p < 2 && e == cudaSuccess; ++p)
        for (int q = 0; q < 2 && e == cudaSuccess; ++q) {
            L->d_split[dir][p][q] = reinterpret_cast<SweepBox*>(mem) + off;
            if (!part[p][q].empty())
                e = cudaMemcpyAsync(L->d_split[dir][p][q], part[p][q].data(), sizeof(SweepBox) * part[p][q].size(),
                                    cudaMemcpyHostToDevice, L->stream);
            off += part[p][q].size();
        }
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "sweep split tables"));
    for (int q = 0; q < 2; ++q) {
        L->split_items[dir][q] = items[q];
        L->split_nboxes[dir][q] = (int)part[0][q].size();
    }
    return BAMREX_OK;
}

extern "C" int bamrex_level_sweep_dir_device_part(bamrex_level* L, int dir, int reduce_ws, int part)
{
    if (!L || dir < 0 || dir >= L->D || part < 0 || part > 1) return fail(BAMREX_ERR_ARG, "bad argument");
    if (!L->run_pending) return L->set_err(fail(BAMREX_ERR_ARG, "call bamrex_level_dist_begin first"));
    if (!L->split_mem[dir]) return L->set_err(fail(BAMREX_ERR_ARG, "call bamrex_level_set_sweep_split first"));
    if (!L->reg_tasks[dir].empty())
        return L->set_err(fail(BAMREX_ERR_UNSUPPORTED, "flux registers are recorded by bamrex_level_advance only"));
    BX_TRY(level_sweep(L, dir, L->cur, 0.0, L->d_scal, reduce_ws != 0, true, part));
    if (part == 1) L->cur ^= 1;  // the direction is complete
    return BAMREX_OK;
}

extern "C" int bamrex_level_dist_end(bamrex_level* L, double* time, double* dt, int* steps)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    if (!L->run_pending) return L->set_err(fail(BAMREX_ERR_ARG, "no run pending"));
    StepScalars* h = L->h_scal;
    cudaError_t e = cudaMemcpyAsync(h, L->d_scal, sizeof(StepScalars), cudaMemcpyDeviceToHost, L->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    L->run_pending = false;
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "split run"));
    // sweeps skipped after the stop time flipped the host's parity too: the
    // result is where the counted steps left it
    if (h->done) L->cur = L->run_start_parity ^ ((h->steps * L->D) & 1);
    L->ws_valid = false;
    if (time) *time = h->time;
    if (dt) *dt = h->dt;
    if (steps) *steps = h->steps;
    if (h->status) return L->set_err(fail(h->status, "non-finite or non-positive time step on the device"));
    return BAMREX_OK;
}
