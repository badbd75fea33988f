// Binary state dump / restore of a 2D AWCM instance (no counterpart in the reference, whose only
// output is the write-only text dump of AWCM_MANAGER_2D::Print, Wavelet/AWCM_MANAGER_2D.h:243-255).
//
// File layout (little-endian), version 1:
//   header, 128 bytes:
//     char     magic[8]       "AWCMST2D"
//     uint32   version         1
//     uint32   header_bytes    128
//     int32    num_levels, nx_coarse, ny_coarse, nx, ny, bc_kind
//     float64  x_min, x_max, y_min, y_max, gamma, t
//     int64    step
//     uint64   n_active        points of mask0 on the Nx x Ny grid
//     uint64   payload_bytes
//     uint32   crc32           CRC-32 (IEEE 802.3, reflected, as zlib) of the payload
//     zero padding to 128 bytes
//   payload:
//     5 mask planes (mask_temp, mask0..mask3) over the ghosted (Ny+6) x (Nx+6) points, one bit
//       per point, least significant bit first, each plane padded to whole bytes;
//     4 level planes (level0..level3) over the Nx x Ny grid points, one signed byte each;
//     the conserved state (rho, rho u, rho v, E) of the mask0 grid points in row-major order
//       (j outer, i inner), 4 doubles each.
// Between steps the state is "values on mask0, zeros elsewhere" (PostProcessEuler), so a restore
// writes zeros at every other point; ghosts are refilled by the boundary fill of the next step.
// The writer and the reader sit on the public C-ABI (awcm2d_get_q / _set_q / masks / levels).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "awcm_b200.h"

namespace awcm {
void set_last_error(const char* msg, const char* file, int line);
}

namespace {

constexpr char kMagic[8] = {'A', 'W', 'C', 'M', 'S', 'T', '2', 'D'};
constexpr uint32_t kVersion = 1;
constexpr uint32_t kHeaderBytes = 128;

struct Header {
    char magic[8];
    uint32_t version, header_bytes;
    int32_t num_levels, nx_coarse, ny_coarse, nx, ny, bc_kind;
    double x_min, x_max, y_min, y_max, gamma, t;
    int64_t step;
    uint64_t n_active, payload_bytes;
    uint32_t crc32;
};
static_assert(sizeof(Header) <= kHeaderBytes, "header fits its 128 bytes");

uint32_t crc32_ieee(const uint8_t* p, size_t n)
{
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t k = 0; k < 256; ++k) {
            uint32_t c = k;
            for (int b = 0; b < 8; ++b) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            table[k] = c;
        }
        init = true;
    }
    uint32_t c = 0xFFFFFFFFu;
    for (size_t k = 0; k < n; ++k) c = table[(c ^ p[k]) & 0xFFu] ^ (c >> 8);
    return c ^ 0xFFFFFFFFu;
}

int fail(int code, const std::string& msg)
{
    awcm::set_last_error(msg.c_str(), __FILE__, __LINE__);
    return code;
}

}  // namespace

extern "C" {

int awcm2d_save_state(awcm2d_t h, const char* path, double t, long long step)
{
    if (!h || !path) return fail(AWCM_ERR_ARG, "null argument");
    int nx = 0, ny = 0;
    awcm2d_geometry gm, *geo = &gm;
    int rc = awcm2d_dims(h, &nx, &ny);
    if (rc || (rc = awcm2d_get_geometry(h, &gm))) return rc;
    const size_t ng = (size_t)(nx + 6) * (ny + 6), ni = (size_t)nx * ny;
    std::vector<double> q(ng * 4);
    std::vector<uint8_t> m(5 * ng);
    std::vector<int> lv(4 * ni);
    if ((rc = awcm2d_get_q(h, q.data())) || (rc = awcm2d_get_masks(h, m.data())) ||
        (rc = awcm2d_get_levels(h, lv.data())))
        return rc;
    const size_t plane_bytes = (ng + 7) / 8;
    std::vector<uint8_t> payload(5 * plane_bytes + 4 * ni, 0);
    for (int p = 0; p < 5; ++p)
        for (size_t k = 0; k < ng; ++k)
            if (m[p * ng + k]) payload[p * plane_bytes + k / 8] |= (uint8_t)(1u << (k % 8));
    uint8_t* lp = payload.data() + 5 * plane_bytes;
    for (size_t k = 0; k < 4 * ni; ++k) lp[k] = (uint8_t)(int8_t)lv[k];
    uint64_t n_active = 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t g = (size_t)(j + 3) * (nx + 6) + (i + 3);
            if (!m[ng + g]) continue;  // mask0 plane
            const size_t at = payload.size();
            payload.resize(at + 4 * sizeof(double));
            std::memcpy(payload.data() + at, &q[g * 4], 4 * sizeof(double));
            ++n_active;
        }
    uint8_t head[kHeaderBytes] = {};
    Header hd{};
    std::memcpy(hd.magic, kMagic, 8);
    hd.version = kVersion;
    hd.header_bytes = kHeaderBytes;
    hd.num_levels = geo->num_levels;
    hd.nx_coarse = geo->nx_coarse;
    hd.ny_coarse = geo->ny_coarse;
    hd.nx = nx;
    hd.ny = ny;
    hd.bc_kind = geo->bc_kind;
    hd.x_min = geo->x_min;
    hd.x_max = geo->x_max;
    hd.y_min = geo->y_min;
    hd.y_max = geo->y_max;
    hd.gamma = geo->gamma;
    hd.t = t;
    hd.step = step;
    hd.n_active = n_active;
    hd.payload_bytes = payload.size();
    hd.crc32 = crc32_ieee(payload.data(), payload.size());
    std::memcpy(head, &hd, sizeof(hd));
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(AWCM_ERR_ARG, std::string("cannot open for writing: ") + path);
    const bool ok = std::fwrite(head, 1, kHeaderBytes, f) == kHeaderBytes &&
                    std::fwrite(payload.data(), 1, payload.size(), f) == payload.size();
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) return fail(AWCM_ERR_ARG, std::string("write failed: ") + path);
    return AWCM_OK;
}

int awcm2d_load_state(awcm2d_t h, const char* path, double* t, long long* step)
{
    if (!h || !path) return fail(AWCM_ERR_ARG, "null argument");
    int nx = 0, ny = 0;
    awcm2d_geometry gm, *geo = &gm;
    int rc = awcm2d_dims(h, &nx, &ny);
    if (rc || (rc = awcm2d_get_geometry(h, &gm))) return rc;
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(AWCM_ERR_ARG, std::string("cannot open: ") + path);
    uint8_t head[kHeaderBytes];
    Header hd{};
    if (std::fread(head, 1, kHeaderBytes, f) != kHeaderBytes) {
        std::fclose(f);
        return fail(AWCM_ERR_STATE, "truncated header");
    }
    std::memcpy(&hd, head, sizeof(hd));
    if (std::memcmp(hd.magic, kMagic, 8) != 0 || hd.version != kVersion || hd.header_bytes != kHeaderBytes) {
        std::fclose(f);
        return fail(AWCM_ERR_STATE, "not an AWCM 2D state file of version 1");
    }
    if (hd.nx != nx || hd.ny != ny || hd.num_levels != geo->num_levels || hd.nx_coarse != geo->nx_coarse ||
        hd.ny_coarse != geo->ny_coarse || hd.bc_kind != geo->bc_kind || hd.x_min != geo->x_min ||
        hd.x_max != geo->x_max || hd.y_min != geo->y_min || hd.y_max != geo->y_max) {
        std::fclose(f);
        return fail(AWCM_ERR_STATE, "state file geometry differs from the instance");
    }
    if (hd.gamma != geo->gamma) {
        // energies and pressures of the stored state belong to another ratio of specific heats
        std::fclose(f);
        return fail(AWCM_ERR_STATE, "state file gamma differs from the instance");
    }
    const size_t ng = (size_t)(nx + 6) * (ny + 6), ni = (size_t)nx * ny, plane_bytes = (ng + 7) / 8;
    const size_t expect = 5 * plane_bytes + 4 * ni + (size_t)hd.n_active * 4 * sizeof(double);
    if (hd.payload_bytes != expect || hd.n_active > ni) {
        std::fclose(f);
        return fail(AWCM_ERR_STATE, "payload size does not match the header");
    }
    std::vector<uint8_t> payload(expect);
    const bool got = std::fread(payload.data(), 1, expect, f) == expect;
    std::fclose(f);
    if (!got) return fail(AWCM_ERR_STATE, "truncated payload");
    if (crc32_ieee(payload.data(), expect) != hd.crc32) return fail(AWCM_ERR_STATE, "payload CRC-32 mismatch");
    std::vector<uint8_t> m(5 * ng);
    for (int p = 0; p < 5; ++p)
        for (size_t k = 0; k < ng; ++k) m[p * ng + k] = (payload[p * plane_bytes + k / 8] >> (k % 8)) & 1u;
    std::vector<int> lv(4 * ni);
    const uint8_t* lp = payload.data() + 5 * plane_bytes;
    for (size_t k = 0; k < 4 * ni; ++k) lv[k] = (int8_t)lp[k];
    std::vector<double> q(ng * 4, 0.0);
    const uint8_t* qp = lp + 4 * ni;
    uint64_t used = 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t g = (size_t)(j + 3) * (nx + 6) + (i + 3);
            if (!m[ng + g]) continue;
            if (used == hd.n_active) return fail(AWCM_ERR_STATE, "more mask0 points than stored values");
            std::memcpy(&q[g * 4], qp + used * 4 * sizeof(double), 4 * sizeof(double));
            ++used;
        }
    if (used != hd.n_active) return fail(AWCM_ERR_STATE, "fewer mask0 points than stored values");
    if ((rc = awcm2d_set_q(h, q.data())) || (rc = awcm2d_set_masks(h, m.data())) ||
        (rc = awcm2d_set_levels(h, lv.data())))
        return rc;
    if (t) *t = hd.t;
    if (step) *step = hd.step;
    return AWCM_OK;
}

}  // extern "C"
