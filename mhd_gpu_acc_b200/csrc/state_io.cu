// state_io.cu -- binary state dump and load (checkpoint / resume).
//
// The reference writes write-only CSV snapshots (scripts/cpu/main_cpu.cpp:36-91)
// and has no reader; a run cannot be resumed.  mhd_state_save writes one grid
// in its own precision, ghost cells included, with the scalars a resumed run
// needs (time, step count, the carried GLM c_h); mhd_state_load reads it back
// into an allocated grid of the same shape and precision, bit for bit.
//
// File layout (little-endian, as the host writes it):
//   bytes   0..7    magic "MHDB200S"
//   bytes   8..11   format version (1)
//   bytes  12..15   dtype (MHD_F64 = 0, MHD_F32 = 1)
//   bytes  16..27   nx, ny, ng (int32)
//   bytes  28..31   zero
//   bytes  32..63   x_min, x_max, y_min, y_max (float64)
//   bytes  64..79   t, ch (float64)
//   bytes  80..87   steps (int64)
//   bytes  88..127  zero
//   bytes 128..     9 planes (rho, rhou, rhov, rhow, Bx, By, Bz, E, psi) of
//                   (ny + 2 ng) rows x (nx + 2 ng) elements, row-major, in the
//                   grid's precision (the grid's row padding is not stored).
// The file is written to "<path>.tmp" and renamed into place, so a reader never
// sees a partial file (the reference's CSV writer does the same,
// scripts/cpu/main_cpu.cpp:36-91).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mhd_b200.h"
#include "launch.h"

namespace mhd {
int report_error(int code, const char* msg);
}

namespace {

constexpr char kMagic[8] = {'M', 'H', 'D', 'B', '2', '0', '0', 'S'};
constexpr uint32_t kVersion = 1;
constexpr size_t kHeader = 128;

int err(int code, const std::string& msg) { return mhd::report_error(code, msg.c_str()); }

bool shape_ok(const mhd_grid* g) {
    return g && g->data && g->nx > 0 && g->ny > 0 && g->ng >= 0 && (g->dtype == MHD_F64 || g->dtype == MHD_F32) &&
           g->pitch >= g->nx + 2LL * g->ng && g->plane >= g->pitch * (g->ny + 2LL * g->ng);
}

}  // namespace

extern "C" int mhd_state_save(const mhd_grid* g, const char* path, const mhd_state_meta* meta) {
    mhd::NvtxRange nvtx_range("mhd_state_save");
    if (!shape_ok(g) || !path) return err(MHD_ERR_ARG, "mhd_state_save: invalid grid or path");
    const size_t es = g->dtype == MHD_F64 ? 8 : 4;
    const size_t tnx = (size_t)g->nx + 2 * g->ng, tny = (size_t)g->ny + 2 * g->ng;
    std::vector<unsigned char> buf(kHeader + (size_t)MHD_NV * tny * tnx * es, 0);
    unsigned char* h = buf.data();
    std::memcpy(h, kMagic, 8);
    const uint32_t ver = kVersion, dt = (uint32_t)g->dtype;
    const int32_t dims[3] = {g->nx, g->ny, g->ng};
    const double ext[4] = {g->x_min, g->x_max, g->y_min, g->y_max};
    const double tc[2] = {meta ? meta->t : 0.0, meta ? meta->ch : 0.0};
    const int64_t steps = meta ? meta->steps : 0;
    std::memcpy(h + 8, &ver, 4);
    std::memcpy(h + 12, &dt, 4);
    std::memcpy(h + 16, dims, 12);
    std::memcpy(h + 32, ext, 32);
    std::memcpy(h + 64, tc, 16);
    std::memcpy(h + 80, &steps, 8);
    for (int f = 0; f < MHD_NV; ++f) {
        const char* src = static_cast<const char*>(g->data) + (size_t)f * g->plane * es;
        const cudaError_t e = cudaMemcpy2D(h + kHeader + (size_t)f * tny * tnx * es, tnx * es, src, g->pitch * es,
                                           tnx * es, tny, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return err(MHD_ERR_CUDA, std::string("mhd_state_save: ") + cudaGetErrorString(e));
    }
    const std::string tmp = std::string(path) + ".tmp";
    FILE* fp = std::fopen(tmp.c_str(), "wb");
    if (!fp) return err(MHD_ERR_ARG, "mhd_state_save: cannot open " + tmp);
    const bool ok = std::fwrite(buf.data(), 1, buf.size(), fp) == buf.size();
    if (std::fclose(fp) != 0 || !ok) {
        std::remove(tmp.c_str());
        return err(MHD_ERR_ARG, "mhd_state_save: write failed for " + tmp);
    }
    if (std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        return err(MHD_ERR_ARG, std::string("mhd_state_save: cannot rename to ") + path);
    }
    return MHD_OK;
}

extern "C" int mhd_state_load(mhd_grid* g, const char* path, mhd_state_meta* meta) {
    mhd::NvtxRange nvtx_range("mhd_state_load");
    if (!shape_ok(g) || !path) return err(MHD_ERR_ARG, "mhd_state_load: invalid grid or path");
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return err(MHD_ERR_ARG, std::string("mhd_state_load: cannot open ") + path);
    unsigned char h[kHeader];
    if (std::fread(h, 1, kHeader, fp) != kHeader || std::memcmp(h, kMagic, 8) != 0) {
        std::fclose(fp);
        return err(MHD_ERR_ARG, std::string("mhd_state_load: not a state file: ") + path);
    }
    uint32_t ver = 0, dt = 0;
    int32_t dims[3];
    std::memcpy(&ver, h + 8, 4);
    std::memcpy(&dt, h + 12, 4);
    std::memcpy(dims, h + 16, 12);
    if (ver != kVersion || (int)dt != g->dtype || dims[0] != g->nx || dims[1] != g->ny || dims[2] != g->ng) {
        std::fclose(fp);
        return err(MHD_ERR_ARG, "mhd_state_load: file version, precision or shape differs from the grid's");
    }
    const size_t es = g->dtype == MHD_F64 ? 8 : 4;
    const size_t tnx = (size_t)g->nx + 2 * g->ng, tny = (size_t)g->ny + 2 * g->ng;
    std::vector<unsigned char> data((size_t)MHD_NV * tny * tnx * es);
    const bool ok = std::fread(data.data(), 1, data.size(), fp) == data.size();
    std::fclose(fp);
    if (!ok) return err(MHD_ERR_ARG, std::string("mhd_state_load: truncated file ") + path);
    for (int f = 0; f < MHD_NV; ++f) {
        char* dst = static_cast<char*>(g->data) + (size_t)f * g->plane * es;
        const cudaError_t e = cudaMemcpy2D(dst, g->pitch * es, data.data() + (size_t)f * tny * tnx * es, tnx * es,
                                           tnx * es, tny, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return err(MHD_ERR_CUDA, std::string("mhd_state_load: ") + cudaGetErrorString(e));
    }
    if (meta) {
        double tc[2];
        int64_t steps;
        std::memcpy(tc, h + 64, 16);
        std::memcpy(&steps, h + 80, 8);
        meta->t = tc[0];
        meta->ch = tc[1];
        meta->steps = steps;
    }
    return MHD_OK;
}
