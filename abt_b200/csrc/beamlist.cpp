// beamlist.cpp -- the beam-list file: per-orientation outbeam lists saved by
// the tracer's host program and replayed through the far-field entry points.
//
// The reference computes an orientation's outbeams (src/beam_loop_mod.f90,
// records of outbeamtype, src/types_mod.f90:8-17) and hands them to
// diff_main at src/pbt_seq_mod.f90:212.  A writer placed at that call site
// appends each orientation to one file; the reader gives back the arrays that
// pbt_diff_batch_c takes.
//
// Layout (little-endian, every section 8-byte aligned):
//   header, 128 B   magic "PBTBEAM1", version, counts (patched at close)
//   grid            theta[ntheta], phi[nphi]                      f64
//   topology        face_off[nfaces+1], face_vi[nface_vi]         i64
//   orientation i   nbeam, next (i64), params_in (144 B),
//                   verts(nverts,3) f64 column-major, nbeam + next outbeam
//                   records (pbt_outbeam, 128 B each)
//   index           file offset of each orientation block          i64
//   trailer, 24 B   index offset, number of orientations, checksum: FNV-1a 64
//                   of the final header followed by the FNV-1a 64 (8 bytes) of
//                   everything between the header and the trailer
// Host-only C++, no device work.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <new>
#include <string>
#include <vector>

#include "pbt_diff.h"
#include "pbt_internal.h"

namespace {

constexpr char kMagic[8] = {'P', 'B', 'T', 'B', 'E', 'A', 'M', '1'};
constexpr uint32_t kVersion = 1;
constexpr int64_t kHeaderBytes = 128;

struct Header {
    char magic[8];
    uint32_t version, header_bytes;
    int64_t norient, nverts, nfaces, nface_vi, ntheta, nphi, nbeam_total, next_total;
    double lambda;
    int64_t reserved[5];
};
static_assert(sizeof(Header) == kHeaderBytes, "header size");
static_assert(sizeof(pbt_outbeam) == 128, "outbeam record size");
static_assert(sizeof(pbt_output_params) == 144, "params record size");

struct Fnv {
    uint64_t h = 1469598103934665603ull;
    void add(const void *p, size_t n) {
        const unsigned char *b = (const unsigned char *)p;
        for (size_t i = 0; i < n; i++) {
            h ^= b[i];
            h *= 1099511628211ull;
        }
    }
};

}  // namespace

struct pbt_beamlist_writer {
    FILE *f = nullptr;
    std::string path;
    Header hd{};
    std::vector<int64_t> index;
    int64_t pos = 0;
    Fnv sum;
    bool failed = false;
    bool put(const void *p, size_t n) {
        if (failed) return false;
        if (n && fwrite(p, 1, n, f) != n) {
            failed = true;
            return false;
        }
        sum.add(p, n);
        pos += (int64_t)n;
        return true;
    }
};

struct pbt_beamlist {
    Header hd{};
    std::vector<double> theta, phi, verts;
    std::vector<int64_t> face_off, face_vi, beam_off, ext_off;
    std::vector<pbt_outbeam> beam, ext;
    std::vector<pbt_output_params> params;
};

using namespace pbt;

extern "C" int pbt_beamlist_writer_open(const char *path, const double *theta, int64_t ntheta,
                                        const double *phi, int64_t nphi, int64_t nverts,
                                        const int64_t *face_off, const int64_t *face_vi,
                                        int64_t nfaces, double lambda,
                                        pbt_beamlist_writer **out) {
    clear_error();
    if (!path || !out || !theta || !phi || !face_off || !face_vi) {
        set_error("beam-list writer: NULL argument");
        return PBT_EINVAL;
    }
    *out = nullptr;
    PBT_TRY(validate_angles(theta, ntheta, phi, nphi));
    if (nverts < 3 || nfaces < 1 || face_off[0] != 0 || !(lambda > 0.0)) {
        set_error("beam-list writer: bad nverts, nfaces, face_off or lambda");
        return PBT_EINVAL;
    }
    for (int64_t i = 0; i < nfaces; i++)
        if (face_off[i + 1] - face_off[i] < 3) {
            set_error("beam-list writer: face %lld has fewer than 3 vertices", (long long)(i + 1));
            return PBT_EINVAL;
        }
    const int64_t nvi = face_off[nfaces];
    for (int64_t i = 0; i < nvi; i++)
        if (face_vi[i] < 1 || face_vi[i] > nverts) {
            set_error("beam-list writer: face vertex index %lld out of range", (long long)face_vi[i]);
            return PBT_EINVAL;
        }
    pbt_beamlist_writer *w = new (std::nothrow) pbt_beamlist_writer;
    if (!w) {
        set_error("beam-list writer: out of host memory");
        return PBT_ENOMEM;
    }
    w->f = fopen(path, "wb");
    if (!w->f) {
        set_error("beam-list writer: cannot open %s", path);
        delete w;
        return PBT_EINVAL;
    }
    w->path = path;
    memcpy(w->hd.magic, kMagic, 8);
    w->hd.version = kVersion;
    w->hd.header_bytes = (uint32_t)kHeaderBytes;
    w->hd.nverts = nverts;
    w->hd.nfaces = nfaces;
    w->hd.nface_vi = nvi;
    w->hd.ntheta = ntheta;
    w->hd.nphi = nphi;
    w->hd.lambda = lambda;
    // the header is rewritten at close; its checksum share is taken then
    Header blank = w->hd;
    bool ok = fwrite(&blank, 1, sizeof(Header), w->f) == sizeof(Header);
    w->pos = kHeaderBytes;
    ok = ok && w->put(theta, ntheta * 8) && w->put(phi, nphi * 8) &&
         w->put(face_off, (nfaces + 1) * 8) && w->put(face_vi, nvi * 8);
    if (!ok) {
        fclose(w->f);
        remove(path);
        delete w;
        set_error("beam-list writer: write failed");
        return PBT_EINVAL;
    }
    *out = w;
    return PBT_OK;
}

extern "C" int pbt_beamlist_writer_add(pbt_beamlist_writer *w, const pbt_outbeam *beam,
                                       int64_t nbeam, const pbt_outbeam *ext, int64_t next,
                                       const double *verts, const pbt_output_params *params_in) {
    clear_error();
    if (!w || !w->f || !verts || !params_in || nbeam < 0 || next < 0 || (nbeam && !beam) ||
        (next && !ext)) {
        set_error("beam-list writer: bad argument");
        return PBT_EINVAL;
    }
    for (int64_t q = 0; q < 3 * w->hd.nverts; q++)
        if (!isfinite(verts[q])) {
            set_error("beam-list writer: non-finite vertex coordinate");
            return PBT_EINVAL;
        }
    for (int64_t i = 0; i < nbeam + next; i++) {
        const pbt_outbeam &ob = i < nbeam ? beam[i] : ext[i - nbeam];
        if (ob.fi < 1 || ob.fi > w->hd.nfaces) {
            set_error("beam-list writer: outbeam %lld has face index %lld (nfaces %lld)",
                      (long long)(i + 1), (long long)ob.fi, (long long)w->hd.nfaces);
            return PBT_EINVAL;
        }
    }
    w->index.push_back(w->pos);
    const int64_t n2[2] = {nbeam, next};
    const bool ok = w->put(n2, 16) && w->put(params_in, sizeof(pbt_output_params)) &&
                    w->put(verts, (size_t)w->hd.nverts * 3 * 8) &&
                    w->put(beam, (size_t)nbeam * sizeof(pbt_outbeam)) &&
                    w->put(ext, (size_t)next * sizeof(pbt_outbeam));
    if (!ok) {
        set_error("beam-list writer: write failed");
        return PBT_EINVAL;
    }
    w->hd.norient++;
    w->hd.nbeam_total += nbeam;
    w->hd.next_total += next;
    return PBT_OK;
}

extern "C" int pbt_beamlist_writer_close(pbt_beamlist_writer *w) {
    clear_error();
    if (!w) return PBT_OK;
    int rc = PBT_OK;
    const int64_t index_at = w->pos;
    bool ok = !w->failed && w->put(w->index.data(), w->index.size() * 8);
    // checksum of the final header followed by the body's hash (the body was
    // hashed while it streamed out; the header is final only now)
    Fnv total;
    total.add(&w->hd, sizeof(Header));
    total.add(&w->sum.h, 8);
    const uint64_t chk = total.h;
    const int64_t tail[2] = {index_at, w->hd.norient};
    ok = ok && fwrite(tail, 1, 16, w->f) == 16 && fwrite(&chk, 1, 8, w->f) == 8;
    ok = ok && fseek(w->f, 0, SEEK_SET) == 0 && fwrite(&w->hd, 1, sizeof(Header), w->f) == sizeof(Header);
    if (fclose(w->f) != 0) ok = false;
    w->f = nullptr;
    if (!ok) {
        set_error("beam-list writer: write failed on %s", w->path.c_str());
        rc = PBT_EINVAL;
    }
    delete w;
    return rc;
}

extern "C" int pbt_beamlist_read(const char *path, pbt_beamlist **out) {
    clear_error();
    if (!path || !out) {
        set_error("beam-list reader: NULL argument");
        return PBT_EINVAL;
    }
    *out = nullptr;
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_error("beam-list reader: cannot open %s", path);
        return PBT_EINVAL;
    }
    std::vector<unsigned char> buf;
    {
        fseek(f, 0, SEEK_END);
        const long n = ftell(f);
        fseek(f, 0, SEEK_SET);
        if (n < kHeaderBytes + 24) {
            fclose(f);
            set_error("beam-list reader: %s is too short to be a beam list", path);
            return PBT_EINVAL;
        }
        buf.resize((size_t)n);
        const size_t got = fread(buf.data(), 1, buf.size(), f);
        fclose(f);
        if (got != buf.size()) {
            set_error("beam-list reader: read failed on %s", path);
            return PBT_EINVAL;
        }
    }
    const int64_t size = (int64_t)buf.size();
    Header hd;
    memcpy(&hd, buf.data(), sizeof(Header));
    if (memcmp(hd.magic, kMagic, 8) != 0) {
        set_error("beam-list reader: %s is not a beam list (bad magic)", path);
        return PBT_EINVAL;
    }
    if (hd.version != kVersion || hd.header_bytes != kHeaderBytes) {
        set_error("beam-list reader: unsupported version %u", hd.version);
        return PBT_EINVAL;
    }
    int64_t tail[2];
    uint64_t chk;
    memcpy(tail, buf.data() + size - 24, 16);
    memcpy(&chk, buf.data() + size - 8, 8);
    {
        Fnv body, total;
        body.add(buf.data() + kHeaderBytes, (size_t)(size - 24 - kHeaderBytes));
        total.add(&hd, sizeof(Header));
        total.add(&body.h, 8);
        if (total.h != chk) {
            set_error("beam-list reader: checksum mismatch in %s (file damaged or truncated)", path);
            return PBT_EINVAL;
        }
    }
    const int64_t no = hd.norient;
    if (tail[1] != no || no < 0 || tail[0] < kHeaderBytes || tail[0] + no * 8 != size - 24 ||
        hd.nverts < 3 || hd.nfaces < 1 || hd.ntheta < 1 || hd.nphi < 1) {
        set_error("beam-list reader: inconsistent counts in %s", path);
        return PBT_EINVAL;
    }
    pbt_beamlist *bl = new (std::nothrow) pbt_beamlist;
    if (!bl) {
        set_error("beam-list reader: out of host memory");
        return PBT_ENOMEM;
    }
    bl->hd = hd;
    int64_t p = kHeaderBytes;
    auto take = [&](void *dst, int64_t n) {
        if (p + n > tail[0]) return false;
        if (n) memcpy(dst, buf.data() + p, (size_t)n);
        p += n;
        return true;
    };
    bl->theta.resize(hd.ntheta);
    bl->phi.resize(hd.nphi);
    bl->face_off.resize(hd.nfaces + 1);
    bl->face_vi.resize(hd.nface_vi);
    bool ok = take(bl->theta.data(), hd.ntheta * 8) && take(bl->phi.data(), hd.nphi * 8) &&
              take(bl->face_off.data(), (hd.nfaces + 1) * 8) &&
              take(bl->face_vi.data(), hd.nface_vi * 8);
    std::vector<int64_t> index(no);
    memcpy(index.data(), buf.data() + tail[0], no * 8);
    bl->beam_off.assign(1, 0);
    bl->ext_off.assign(1, 0);
    bl->verts.resize((size_t)no * hd.nverts * 3);
    bl->params.resize(no);
    bl->beam.reserve(hd.nbeam_total);
    bl->ext.reserve(hd.next_total);
    for (int64_t o = 0; ok && o < no; o++) {
        p = index[o];
        int64_t n2[2];
        ok = p >= kHeaderBytes && take(n2, 16) && n2[0] >= 0 && n2[1] >= 0 &&
             take(&bl->params[o], sizeof(pbt_output_params)) &&
             take(bl->verts.data() + (size_t)o * hd.nverts * 3, hd.nverts * 3 * 8);
        if (!ok) break;
        const size_t b0 = bl->beam.size(), e0 = bl->ext.size();
        if (p + (n2[0] + n2[1]) * (int64_t)sizeof(pbt_outbeam) > tail[0]) {
            ok = false;
            break;
        }
        bl->beam.resize(b0 + n2[0]);
        bl->ext.resize(e0 + n2[1]);
        ok = take(bl->beam.data() + b0, n2[0] * sizeof(pbt_outbeam)) &&
             take(bl->ext.data() + e0, n2[1] * sizeof(pbt_outbeam));
        bl->beam_off.push_back((int64_t)bl->beam.size());
        bl->ext_off.push_back((int64_t)bl->ext.size());
    }
    if (!ok || (int64_t)bl->beam.size() != hd.nbeam_total || (int64_t)bl->ext.size() != hd.next_total) {
        delete bl;
        set_error("beam-list reader: %s has a damaged orientation block", path);
        return PBT_EINVAL;
    }
    *out = bl;
    return PBT_OK;
}

extern "C" int pbt_beamlist_info(const pbt_beamlist *bl, int64_t counts[8], double *lambda) {
    clear_error();
    if (!bl || !counts) {
        set_error("beam-list: NULL argument");
        return PBT_EINVAL;
    }
    const Header &h = bl->hd;
    const int64_t c[8] = {h.norient, h.nverts, h.nfaces, h.nface_vi,
                          h.ntheta,  h.nphi,   h.nbeam_total, h.next_total};
    memcpy(counts, c, sizeof(c));
    if (lambda) *lambda = h.lambda;
    return PBT_OK;
}

extern "C" int pbt_beamlist_arrays(const pbt_beamlist *bl, const double **theta, const double **phi,
                                   const int64_t **face_off, const int64_t **face_vi,
                                   const double **verts, const int64_t **beam_off,
                                   const pbt_outbeam **beam, const int64_t **ext_off,
                                   const pbt_outbeam **ext, const pbt_output_params **params_in) {
    clear_error();
    if (!bl) {
        set_error("beam-list: NULL argument");
        return PBT_EINVAL;
    }
    if (theta) *theta = bl->theta.data();
    if (phi) *phi = bl->phi.data();
    if (face_off) *face_off = bl->face_off.data();
    if (face_vi) *face_vi = bl->face_vi.data();
    if (verts) *verts = bl->verts.data();
    if (beam_off) *beam_off = bl->beam_off.data();
    if (beam) *beam = bl->beam.data();
    if (ext_off) *ext_off = bl->ext_off.data();
    if (ext) *ext = bl->ext.data();
    if (params_in) *params_in = bl->params.data();
    return PBT_OK;
}

extern "C" int pbt_beamlist_free(pbt_beamlist *bl) {
    delete bl;
    return PBT_OK;
}
