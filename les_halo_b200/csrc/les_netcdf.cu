// les_netcdf.cu -- the NetCDF output of the reference's OpenCL host
// (src/OpenCL/module_LES_write_netcdf.f95), host code only.
//
// Six files as init_netcdf_file (:105-322) creates them: LES_output.nc and
// LES_output_p.nc (pressure), LES_output_u/_v/_w.nc (velocity_x/_y/_z) and
// LES_output_uvwsum.nc (velocity_sum_x/_y/_z).  Each has the dimensions
// level, latitude, longitude (the full Fortran extents of its arrays,
// ghosts included) and time (a fixed length, NTIMESTEPS = 20 in the
// reference), coordinate variables latitude and longitude (FP32, 1..n) and
// time (FP64, 1..ntimes) with units attributes, and the data variables
// (FP32, dims (time, level, latitude, longitude), unit attribute).
// write_to_netcdf_file (:324-357) puts one time slab of the whole arrays.
//
// Written directly in the published classic format (big-endian header of
// dimension, attribute and variable lists, then each variable's data at its
// offset): version 1 (32-bit offsets) while the file stays below 2 GiB,
// else the 64-bit-offset version 2 (always, with LES_NETCDF_64BIT=1).  Time
// slabs never written hold the default float fill value, as the library's
// fill mode leaves them.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "les_abi.h"
#include "les_nvtx.h"

les_status les_internal_fail(les_status s, const char *msg);
les_status les_internal_ok();

namespace {

constexpr uint32_t kNcDimension = 0x0A, kNcVariable = 0x0B, kNcAttribute = 0x0C;
constexpr uint32_t kNcChar = 2, kNcFloat = 5, kNcDouble = 6;
constexpr float kFillFloat = 9.9692099683868690e+36f;

les_status nc_fail(les_status s, const std::string &m) { return les_internal_fail(s, m.c_str()); }

struct NcVar {
    std::string name, units;
    std::vector<uint32_t> dims;
    uint32_t type;
    uint64_t vsize = 0, begin = 0;
};

struct NcFile {
    std::string path;
    FILE *fp = nullptr;
    uint32_t nlvl = 0, nlat = 0, nlon = 0, ntime = 0;
    std::vector<NcVar> vars;  // latitude, longitude, time, data variables
    int ndata = 0;
    std::vector<char> written;  // [data var][time]
    int version = 1;
    uint64_t slab() const { return (uint64_t)nlvl * nlat * nlon * 4; }
};

struct Buf {
    std::vector<unsigned char> b;
    void u32(uint32_t x) {
        for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(x >> s));
    }
    void u64(uint64_t x) {
        for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(x >> s));
    }
    void str(const std::string &s) {  // nelems, chars, zero padding to 4 bytes
        u32((uint32_t)s.size());
        b.insert(b.end(), s.begin(), s.end());
        while (b.size() % 4) b.push_back(0);
    }
};

void header(const NcFile &f, Buf &h) {
    h.b = {'C', 'D', 'F', (unsigned char)f.version};
    h.u32(0);  // numrecs: no record dimension
    const char *dn[4] = {"level", "latitude", "longitude", "time"};
    const uint32_t dl[4] = {f.nlvl, f.nlat, f.nlon, f.ntime};
    h.u32(kNcDimension);
    h.u32(4);
    for (int d = 0; d < 4; ++d) {
        h.str(dn[d]);
        h.u32(dl[d]);
    }
    h.u32(0);  // no global attributes
    h.u32(0);
    h.u32(kNcVariable);
    h.u32((uint32_t)f.vars.size());
    for (const NcVar &v : f.vars) {
        h.str(v.name);
        h.u32((uint32_t)v.dims.size());
        for (uint32_t d : v.dims) h.u32(d);
        h.u32(kNcAttribute);
        h.u32(1);
        h.str("units");
        h.u32(kNcChar);
        h.str(v.units);
        h.u32(v.type);
        h.u32(v.vsize >= 0xffffffffull ? 0xffffffffu : (uint32_t)v.vsize);
        if (f.version == 1)
            h.u32((uint32_t)v.begin);
        else
            h.u64(v.begin);
    }
}

les_status put_at(NcFile &f, uint64_t off, const void *data, size_t bytes) {
    if (fseeko(f.fp, (off_t)off, SEEK_SET) != 0 || std::fwrite(data, 1, bytes, f.fp) != bytes)
        return nc_fail(LES_ERR_IO, f.path + ": write failed");
    return LES_OK;
}

// n 4-byte items (FP32) or 8-byte items (FP64), big-endian, at off.
les_status put_be(NcFile &f, uint64_t off, const void *items, size_t n, size_t w) {
    std::vector<unsigned char> out(n * w);
    const unsigned char *in = static_cast<const unsigned char *>(items);
    for (size_t q = 0; q < n; ++q)
        for (size_t b = 0; b < w; ++b) out[q * w + b] = in[q * w + (w - 1 - b)];
    return put_at(f, off, out.data(), out.size());
}

les_status nc_create(NcFile &f, const std::string &path, uint32_t nlvl, uint32_t nlat, uint32_t nlon, uint32_t ntime,
                     const std::vector<std::pair<std::string, std::string>> &data) {
    f.path = path;
    f.nlvl = nlvl;
    f.nlat = nlat;
    f.nlon = nlon;
    f.ntime = ntime;
    f.vars = {NcVar{"latitude", "degrees_north", {1}, kNcFloat},
              NcVar{"longitude", "degrees_east", {2}, kNcFloat},
              NcVar{"time", "hours since 2014-08-05 16:00:00", {3}, kNcDouble}};
    for (const auto &d : data) f.vars.push_back(NcVar{d.first, d.second, {3, 0, 1, 2}, kNcFloat});
    f.ndata = (int)data.size();
    f.vars[0].vsize = 4ull * nlat;
    f.vars[1].vsize = 4ull * nlon;
    f.vars[2].vsize = 8ull * ntime;
    for (int q = 3; q < (int)f.vars.size(); ++q) f.vars[q].vsize = f.slab() * ntime;
    for (size_t q = 0; q < f.vars.size(); ++q) f.vars[q].vsize = (f.vars[q].vsize + 3) / 4 * 4;
    // offsets: the header length does not depend on them beyond their width
    const char *force = std::getenv("LES_NETCDF_64BIT");
    for (f.version = (force && force[0] == '1') ? 2 : 1;; f.version = 2) {
        Buf h;
        header(f, h);
        uint64_t off = h.b.size();
        for (NcVar &v : f.vars) {
            v.begin = off;
            off += v.vsize;
        }
        if (f.version == 2 || off < (1ull << 31)) break;
    }
    for (size_t q = 0; q + 1 < f.vars.size(); ++q)
        if (f.vars[q].vsize >= 0xffffffffull)
            return nc_fail(LES_ERR_DIMS, path + ": a variable other than the last exceeds 4 GiB");
    f.fp = std::fopen(path.c_str(), "wb");
    if (!f.fp) return nc_fail(LES_ERR_IO, path + ": cannot open for writing");
    Buf h;
    header(f, h);
    les_status s = put_at(f, 0, h.b.data(), h.b.size());
    if (s != LES_OK) return s;
    std::vector<float> lat(nlat), lon(nlon);
    std::vector<double> tm(ntime);
    for (uint32_t q = 0; q < nlat; ++q) lat[q] = (float)(q + 1);
    for (uint32_t q = 0; q < nlon; ++q) lon[q] = (float)(q + 1);
    for (uint32_t q = 0; q < ntime; ++q) tm[q] = (double)(float)(q + 1);
    if ((s = put_be(f, f.vars[0].begin, lat.data(), nlat, 4)) != LES_OK) return s;
    if ((s = put_be(f, f.vars[1].begin, lon.data(), nlon, 4)) != LES_OK) return s;
    if ((s = put_be(f, f.vars[2].begin, tm.data(), ntime, 8)) != LES_OK) return s;
    f.written.assign((size_t)f.ndata * ntime, 0);
    return LES_OK;
}

les_status nc_put_slab(NcFile &f, int var, int t, const float *a) {
    const NcVar &v = f.vars[3 + var];
    les_status s = put_be(f, v.begin + (uint64_t)(t - 1) * f.slab(), a, (size_t)(f.slab() / 4), 4);
    if (s == LES_OK) f.written[(size_t)var * f.ntime + (t - 1)] = 1;
    return s;
}

// Fill the slabs never written, then close.
les_status nc_close(NcFile &f) {
    if (!f.fp) return LES_OK;
    les_status s = LES_OK;
    std::vector<float> fill;
    for (int var = 0; var < f.ndata && s == LES_OK; ++var)
        for (uint32_t t = 1; t <= f.ntime && s == LES_OK; ++t)
            if (!f.written[(size_t)var * f.ntime + (t - 1)]) {
                if (fill.empty()) fill.assign((size_t)(f.slab() / 4), kFillFloat);
                s = nc_put_slab(f, var, (int)t, fill.data());
            }
    if (std::fclose(f.fp) != 0 && s == LES_OK) s = nc_fail(LES_ERR_IO, f.path + ": close failed");
    f.fp = nullptr;
    return s;
}

}  // namespace

struct les_netcdf {
    int ip = 0, jp = 0, kp = 0, ntimes = 0;
    NcFile f[6];  // LES_output, _p, _u, _v, _w, _uvwsum
};

extern "C" {

les_status les_netcdf_open(const char *prefix, int ip, int jp, int kp, int ntimes, les_netcdf **out) {
    LES_RANGE("les_netcdf_open");
    if (!out) return les_internal_fail(LES_ERR_BAD_ARG, "NULL handle");
    *out = nullptr;
    if (ip < 1 || jp < 1 || kp < 1 || ntimes < 1) return les_internal_fail(LES_ERR_BAD_ARG, "bad grid or time count");
    const std::string pre = prefix ? prefix : "./";
    les_netcdf *nc = new les_netcdf();
    nc->ip = ip;
    nc->jp = jp;
    nc->kp = kp;
    nc->ntimes = ntimes;
    const uint32_t T = (uint32_t)ntimes;
    const std::pair<std::string, std::string> pres{"pressure", "hPa"};
    les_status s = nc_create(nc->f[0], pre + "LES_output.nc", kp + 2, jp + 3, ip + 3, T, {pres});
    if (s == LES_OK) s = nc_create(nc->f[1], pre + "LES_output_p.nc", kp + 2, jp + 3, ip + 3, T, {pres});
    if (s == LES_OK)
        s = nc_create(nc->f[2], pre + "LES_output_u.nc", kp + 2, jp + 3, ip + 2, T, {{"velocity_x", "m/s"}});
    if (s == LES_OK)
        s = nc_create(nc->f[3], pre + "LES_output_v.nc", kp + 2, jp + 3, ip + 2, T, {{"velocity_y", "m/s"}});
    if (s == LES_OK)
        s = nc_create(nc->f[4], pre + "LES_output_w.nc", kp + 3, jp + 3, ip + 2, T, {{"velocity_z", "m/s"}});
    if (s == LES_OK)
        s = nc_create(nc->f[5], pre + "LES_output_uvwsum.nc", kp + 1, jp + 1, ip + 1, T,
                      {{"velocity_sum_x", "m/s"}, {"velocity_sum_y", "m/s"}, {"velocity_sum_z", "m/s"}});
    if (s != LES_OK) {
        for (NcFile &f : nc->f)
            if (f.fp) std::fclose(f.fp);
        delete nc;
        return s;
    }
    *out = nc;
    return les_internal_ok();
}

les_status les_netcdf_write_host(les_netcdf *nc, int t, const float *p, const float *u, const float *v,
                                 const float *w, const float *usum, const float *vsum, const float *wsum) {
    LES_RANGE("les_netcdf_write_host");
    if (!nc || !p || !u || !v || !w || !usum || !vsum || !wsum)
        return les_internal_fail(LES_ERR_BAD_ARG, "NULL argument");
    if (t < 1 || t > nc->ntimes) {
        char m[128];
        std::snprintf(m, sizeof m, "time index %d outside 1..%d of the time dimension", t, nc->ntimes);
        return les_internal_fail(LES_ERR_BAD_ARG, m);
    }
    les_status s = nc_put_slab(nc->f[0], 0, t, p);
    if (s == LES_OK) s = nc_put_slab(nc->f[1], 0, t, p);
    if (s == LES_OK) s = nc_put_slab(nc->f[2], 0, t, u);
    if (s == LES_OK) s = nc_put_slab(nc->f[3], 0, t, v);
    if (s == LES_OK) s = nc_put_slab(nc->f[4], 0, t, w);
    if (s == LES_OK) s = nc_put_slab(nc->f[5], 0, t, usum);
    if (s == LES_OK) s = nc_put_slab(nc->f[5], 1, t, vsum);
    if (s == LES_OK) s = nc_put_slab(nc->f[5], 2, t, wsum);
    return s == LES_OK ? les_internal_ok() : s;
}

les_status les_netcdf_write(les_netcdf *nc, les_ctx *ctx, int t) {
    LES_RANGE("les_netcdf_write");
    if (!nc || !ctx) return les_internal_fail(LES_ERR_BAD_ARG, "NULL argument");
    const size_t ip = nc->ip, jp = nc->jp, kp = nc->kp;
    std::vector<float> p((ip + 3) * (jp + 3) * (kp + 2)), u((ip + 2) * (jp + 3) * (kp + 2)), v(u.size()),
        w((ip + 2) * (jp + 3) * (kp + 3)), us((ip + 1) * (jp + 1) * (kp + 1)), vs(us.size()), ws(us.size());
    les_host_fields hf;
    std::memset(&hf, 0, sizeof hf);
    hf.p = p.data();
    hf.u = u.data();
    hf.v = v.data();
    hf.w = w.data();
    hf.usum = us.data();
    hf.vsum = vs.data();
    hf.wsum = ws.data();
    les_status s = les_ctx_download(ctx, &hf);
    if (s != LES_OK) return s;
    return les_netcdf_write_host(nc, t, p.data(), u.data(), v.data(), w.data(), us.data(), vs.data(), ws.data());
}

les_status les_netcdf_close(les_netcdf *nc) {
    LES_RANGE("les_netcdf_close");
    if (!nc) return les_internal_ok();
    les_status s = LES_OK;
    for (NcFile &f : nc->f) {
        const les_status q = nc_close(f);
        if (s == LES_OK) s = q;
    }
    delete nc;
    return s == LES_OK ? les_internal_ok() : s;
}

}  // extern "C"
