// Peel-off imaging of the ionizing/FUV band (ion_peel_mod.f90): the
// observers and the image plane at set-up (ion_peel_setup, :49-206), the
// images of the imaging pass on the device (the kernels are the walk
// kernels' peel_direct / peel_scatter in transport.cu), and the image file
// (ion_peel_write, :359-523) in the format of the rates file: a directory
// <base>_image/ with one .npy per image block and header.json.
#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "ctx.h"
#include "mochii_gpu.h"
#include "physics.cuh"

namespace mochii {

namespace {
constexpr double kD2R = kPi / 180.0, kR2D = 180.0 / kPi;
bool fin(double x) { return std::isfinite(x); }
}  // namespace

// ion_peel_setup: observers from the angle lists (alpha, beta, gamma; the
// phase / inclination / position angles are their negatives) or from the
// positions obsx/y/z, default one observer on the +z axis at 1e3 box
// half-widths; the grid -> observer rotation; pixel sizes that frame the
// whole box when dxim/dyim are unset.  Fills c->peel_obs (kPeelObs per
// observer) and c->par's derived distance, dxim, dyim, and allocates the
// device copies and images.
cudaError_t peel_setup(mochii_ctx* c) {
    mochii_params& p = c->par;
    c->peel_obs.clear();
    if (!p.ion_peel) return cudaSuccess;
    for (int i = 0; i < MOCHII_MAX_OBS; ++i) {
        if (fin(p.phase_angle[i])) p.alpha[i] = -p.phase_angle[i];
        if (fin(p.inclination_angle[i])) p.beta[i] = -p.inclination_angle[i];
        if (fin(p.position_angle[i])) p.gamma[i] = -p.position_angle[i];
        if (fin(p.beta[i]) && !fin(p.alpha[i])) p.alpha[i] = 0.0;
        if (fin(p.alpha[i]) && !fin(p.beta[i])) p.beta[i] = 0.0;
    }
    const double xm = std::max({c->grid.xmax, c->grid.ymax, c->grid.zmax});
    const bool by_angle = fin(p.alpha[0]) && fin(p.beta[0]);
    if (!by_angle && !(fin(p.obsx[0]) && fin(p.obsy[0]) && fin(p.obsz[0]))) {
        if (!fin(p.distance)) p.distance = xm * 1.0e3;
        p.obsx[0] = 0.0; p.obsy[0] = 0.0; p.obsz[0] = p.distance;
        p.alpha[0] = 0.0; p.beta[0] = 0.0;
    }
    struct Angles { double ca, sa, cb, sb, cg, sg; };
    std::vector<Angles> ang;
    std::vector<double> pos, tri;   // x, y, z and alpha, beta, gamma per observer
    if (fin(p.alpha[0]) && fin(p.beta[0])) {
        if (!fin(p.distance)) p.distance = xm * 1.0e3;
        for (int i = 0; i < MOCHII_MAX_OBS; ++i) {
            if (!(fin(p.alpha[i]) && fin(p.beta[i]))) continue;
            if (!fin(p.gamma[i])) p.gamma[i] = p.beta[i] > 0.0 && p.beta[i] <= 90.0 ? 90.0 : p.beta[i] > 90.0 ? -90.0 : 0.0;
            Angles a{std::cos(p.alpha[i] * kD2R), std::sin(p.alpha[i] * kD2R), std::cos(p.beta[i] * kD2R),
                     std::sin(p.beta[i] * kD2R), std::cos(p.gamma[i] * kD2R), std::sin(p.gamma[i] * kD2R)};
            ang.push_back(a);
            pos.insert(pos.end(), {p.distance * a.ca * a.sb, p.distance * a.sa * a.sb, p.distance * a.cb});
            tri.insert(tri.end(), {p.alpha[i], p.beta[i], p.gamma[i]});
        }
    } else {
        if (!fin(p.distance)) {
            p.distance = std::sqrt(p.obsx[0] * p.obsx[0] + p.obsy[0] * p.obsy[0] + p.obsz[0] * p.obsz[0]);
            if (p.distance < 10.0 * xm) p.distance = xm * 1.0e3;
        }
        for (int i = 0; i < MOCHII_MAX_OBS; ++i) {
            if (!(fin(p.obsx[i]) && fin(p.obsy[i]) && fin(p.obsz[i]))) continue;
            if (!fin(p.gamma[i])) p.gamma[i] = 0.0;
            const double robs = std::sqrt(p.obsx[i] * p.obsx[i] + p.obsy[i] * p.obsy[i] + p.obsz[i] * p.obsz[i]);
            const double scale = p.distance / robs;
            const double ox = scale > 1.001 ? p.obsx[i] * scale : p.obsx[i];
            const double oy = scale > 1.001 ? p.obsy[i] * scale : p.obsy[i];
            const double oz = scale > 1.001 ? p.obsz[i] * scale : p.obsz[i];
            // the direction cosine from the observer's own radius
            const double cb = std::min(std::max(robs > 0.0 ? p.obsz[i] / robs : 1.0, -1.0), 1.0);
            const double sb = std::sqrt(1.0 - cb * cb);
            p.beta[i] = std::atan2(sb, cb) * kR2D;
            double ca = 1.0, sa = 0.0;
            if (sb == 0.0) {
                p.alpha[i] = 0.0;
            } else {
                const double al = std::atan2(oy, ox);
                ca = std::cos(al);
                sa = std::sin(al);
                p.alpha[i] = al * kR2D;
            }
            ang.push_back(Angles{ca, sa, cb, sb, std::cos(p.gamma[i] * kD2R), std::sin(p.gamma[i] * kD2R)});
            pos.insert(pos.end(), {ox, oy, oz});
            tri.insert(tri.end(), {p.alpha[i], p.beta[i], p.gamma[i]});
        }
    }
    if (!(fin(p.dxim) && fin(p.dyim))) {
        p.dxim = std::atan2(xm * std::sqrt(3.0), p.distance) / (p.nxim / 2.0) * kR2D;
        p.dyim = std::atan2(xm * std::sqrt(3.0), p.distance) / (p.nyim / 2.0) * kR2D;
    }
    const int nobs = (int)ang.size();
    for (int k = 0; k < nobs; ++k) {
        const Angles& a = ang[k];
        const double R[9] = {a.ca * a.cb * a.cg - a.sa * a.sg, a.sa * a.cb * a.cg + a.ca * a.sg, -a.sb * a.cg,
                             -a.ca * a.cb * a.sg - a.sa * a.cg, -a.sa * a.cb * a.sg + a.ca * a.cg, a.sb * a.sg,
                             a.ca * a.sb, a.sa * a.sb, a.cb};
        const double o[9] = {pos[3 * k], pos[3 * k + 1], pos[3 * k + 2], tri[3 * k], tri[3 * k + 1], tri[3 * k + 2],
                             p.distance, p.dxim, p.dyim};
        c->peel_obs.insert(c->peel_obs.end(), o, o + 9);
        c->peel_obs.insert(c->peel_obs.end(), R, R + 9);
    }
    // channels: one per band bin with peel_bins, else ionizing (0) and FUV (1, below eion_min)
    const int nnu = c->nnu;
    const int nchan = p.peel_bins ? nnu : (p.add_fuv ? 2 : 1);
    std::vector<int> chan(nnu);
    for (int i = 0; i < nnu; ++i) {
        const double ec = std::sqrt(c->band.eedge[i] * c->band.eedge[i + 1]);
        chan[i] = p.peel_bins ? i : (nchan == 2 && ec < p.eion_min ? 1 : 0);
    }
    const size_t npix = (size_t)nobs * nchan * p.nxim * p.nyim;
    const size_t bytes = c->peel_obs.size() * 8 + (size_t)nnu * 4 + 16 + npix * 8 * (p.save_direc0 ? 3 : 2);
    cudaError_t e = cudaMalloc(&c->peel_blob, bytes);
    if (e != cudaSuccess) return e;
    unsigned char* b = static_cast<unsigned char*>(c->peel_blob);
    PeelDev& d = c->peel;
    d.nobs = nobs;
    d.nchan = nchan;
    d.nxim = p.nxim;
    d.nyim = p.nyim;
    d.direc0 = p.save_direc0 ? 1 : 0;
    double* imgs = reinterpret_cast<double*>(b);
    d.img_dir = imgs;
    d.img_sca = imgs + npix;
    d.img_dir0 = p.save_direc0 ? imgs + 2 * npix : nullptr;
    double* obs = imgs + npix * (p.save_direc0 ? 3 : 2);
    d.obs = obs;
    int* ch = reinterpret_cast<int*>(obs + c->peel_obs.size());
    d.chan = ch;
    if ((e = cudaMemcpy(obs, c->peel_obs.data(), c->peel_obs.size() * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if ((e = cudaMemcpy(ch, chan.data(), (size_t)nnu * 4, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    return cudaMemset(imgs, 0, npix * 8 * (p.save_direc0 ? 3 : 2));
}

// Zero the images before an imaging pass.
cudaError_t peel_clear(mochii_ctx* c) {
    const size_t npix = (size_t)c->peel.nobs * c->peel.nchan * c->peel.nxim * c->peel.nyim;
    return cudaMemsetAsync(c->peel.img_dir, 0, npix * 8 * (c->peel.direc0 ? 3 : 2), c->stream);
}

}  // namespace mochii

using namespace mochii;

extern "C" int mochii_image_shape(const mochii_ctx* c, int* shape4) {
    if (!c || !shape4) return MOCHII_ERR_BAD_PARAM;
    shape4[0] = c->peel.nobs;
    shape4[1] = c->peel.nchan;
    shape4[2] = c->peel.nyim;
    shape4[3] = c->peel.nxim;
    return MOCHII_OK;
}

extern "C" int mochii_image_observer(const mochii_ctx* c, int k, double* out18) {
    if (!c || !out18 || k < 0 || k >= c->peel.nobs) return MOCHII_ERR_BAD_PARAM;
    std::memcpy(out18, c->peel_obs.data() + (size_t)k * kPeelObs, kPeelObs * sizeof(double));
    return MOCHII_OK;
}

extern "C" int mochii_get_image(mochii_ctx* c, int which, double* out, int64_t n) {
    if (!c || !out) return MOCHII_ERR_BAD_PARAM;
    const PeelDev& d = c->peel;
    const long long npix = (long long)d.nobs * d.nchan * d.nyim * d.nxim;
    if (npix == 0 || n != npix) {
        c->last_error = "mochii_get_image: size mismatch or par%ion_peel off";
        return MOCHII_ERR_BAD_PARAM;
    }
    const double* src = which == 0 ? d.img_dir : which == 1 ? d.img_sca : which == 2 ? d.img_dir0 : nullptr;
    if (!src) {
        c->last_error = "mochii_get_image: which is 0 (direct), 1 (scattered) or 2 (unattenuated, save_direc0)";
        return MOCHII_ERR_BAD_PARAM;
    }
    if (cudaMemcpyAsync(out, src, (size_t)npix * 8, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return MOCHII_ERR_CUDA;
    return MOCHII_OK;
}

namespace {
bool npy_write(const std::string& path, const std::vector<long long>& shape, const double* v, size_t n) {
    std::string sh = "(";
    for (size_t i = 0; i < shape.size(); ++i) sh += std::to_string(shape[i]) + (shape.size() == 1 ? "," : i + 1 < shape.size() ? ", " : "");
    sh += ")";
    std::string hdr = "{'descr': '<f8', 'fortran_order': False, 'shape': " + sh + ", }";
    const size_t pad = (64 - (10 + hdr.size() + 1) % 64) % 64;
    hdr += std::string(pad, ' ') + "\n";
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
    const unsigned short hl = (unsigned short)hdr.size();
    bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(&hl, 2, 1, f) == 1 &&
              std::fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size() && std::fwrite(v, 8, n, f) == n;
    return std::fclose(f) == 0 && ok;
}
std::string num(double x) {
    char b[40];
    std::snprintf(b, sizeof(b), "%.17g", x);
    return std::isfinite(x) ? std::string(b) : std::string("null");
}
}  // namespace

// ion_peel_write: surface brightness [erg/s/cm^2/sr] = the accumulated
// contributions / (distance2cm^2 x pixel solid angle).
extern "C" int mochii_write_image(mochii_ctx* c, const char* base) {
    if (!c || !base || !base[0]) return MOCHII_ERR_BAD_PARAM;
    const PeelDev& d = c->peel;
    if (d.nobs == 0) {
        c->last_error = "mochii_write_image: par%ion_peel is off";
        return MOCHII_ERR_BAD_PARAM;
    }
    const mochii_params& p = c->par;
    const long long nimg = (long long)d.nyim * d.nxim, npix = (long long)d.nobs * d.nchan * nimg;
    std::vector<double> dir((size_t)npix), sca((size_t)npix), dir0(d.direc0 ? (size_t)npix : 0);
    int rc = mochii_get_image(c, 0, dir.data(), npix);
    if (!rc) rc = mochii_get_image(c, 1, sca.data(), npix);
    if (!rc && d.direc0) rc = mochii_get_image(c, 2, dir0.data(), npix);
    if (rc) return rc;
    const std::string dir_name = std::string(base) + "_image";
    if (::mkdir(dir_name.c_str(), 0755) != 0 && errno != EEXIST) {
        c->last_error = "mochii_write_image: cannot create " + dir_name;
        return MOCHII_ERR_BAD_PARAM;
    }
    std::string entries;
    auto put = [&](const std::string& ext, const std::vector<long long>& shape, const double* v, size_t n,
                   const std::string& comment, const std::string& kw) -> bool {
        if (!npy_write(dir_name + "/" + ext + ".npy", shape, v, n)) return false;
        std::string sh = "[";
        for (size_t i = 0; i < shape.size(); ++i) sh += std::to_string(shape[i]) + (i + 1 < shape.size() ? ", " : "");
        entries += std::string(entries.empty() ? "" : ",\n") + "    {\"EXTNAME\": \"" + ext + "\", \"file\": \"" + ext +
                   ".npy\", \"shape\": " + sh + "], \"comment\": \"" + comment + "\"" + (kw.empty() ? "" : ", " + kw) + "}";
        return true;
    };
    const char* chname[2] = {"ion", "fuv"};
    const int nnu = c->nnu;
    std::vector<double> ebin(nnu), dbin(nnu), wl(nnu);
    for (int i = 0; i < nnu; ++i) {
        ebin[i] = std::sqrt(c->band.eedge[i] * c->band.eedge[i + 1]);
        dbin[i] = c->band.eedge[i + 1] - c->band.eedge[i];
        wl[i] = 12398.4198 / ebin[i];
    }
    bool ok = true;
    for (int k = 0; k < d.nobs && ok; ++k) {
        const double* o = c->peel_obs.data() + (size_t)k * kPeelObs;
        const double sr = p.dxim * p.dyim * kD2R * kD2R;
        const double fac = 1.0 / (p.distance2cm * p.distance2cm * sr);
        const std::string suf = d.nobs > 1 ? "_obs" + std::to_string(k + 1) : "";
        const std::string kw = "\"DXIM\": " + num(p.dxim) + ", \"DIST\": " + num(o[6]) + ", \"ALPHA\": " + num(o[3]) +
                               ", \"BETA\": " + num(o[4]) + ", \"GAMMA\": " + num(o[5]);
        auto scaled = [&](const std::vector<double>& src, int ch) {
            std::vector<double> v((size_t)nimg);
            for (long long q = 0; q < nimg; ++q) v[q] = src[((size_t)k * d.nchan + ch) * nimg + q] * fac;
            return v;
        };
        if (p.peel_bins) {   // bin-resolved cubes, then the band-integrated channels derived from them
            std::vector<double> cube((size_t)nnu * nimg);
            const std::vector<double>* srcs[3] = {&dir, &sca, &dir0};
            const char* cname[3] = {"direct_cube", "scatt_cube", "direc0_cube"};
            for (int s = 0; s < (d.direc0 ? 3 : 2) && ok; ++s) {
                for (int b = 0; b < nnu; ++b) {
                    const std::vector<double> v = scaled(*srcs[s], b);
                    std::copy(v.begin(), v.end(), cube.begin() + (size_t)b * nimg);
                }
                ok = put(cname[s] + suf, {nnu, d.nyim, d.nxim}, cube.data(), cube.size(), "I(x,y,bin) [erg/s/cm^2/sr]", kw);
            }
            if (k == 0 && ok) {
                ok = put("E_bin", {nnu}, ebin.data(), nnu, "band bin center [eV]", "") &&
                     put("dE_bin", {nnu}, dbin.data(), nnu, "band bin width [eV]", "") &&
                     put("wl_bin", {nnu}, wl.data(), nnu, "band bin center [Angstrom]", "");
            }
            for (int ich = 0; ich < (p.add_fuv ? 2 : 1) && ok; ++ich) {
                for (int s = 0; s < (d.direc0 ? 3 : 2) && ok; ++s) {
                    std::vector<double> img((size_t)nimg, 0.0);
                    for (int b = 0; b < nnu; ++b) {
                        if ((ich == 0) != (ebin[b] >= p.eion_min)) continue;
                        const std::vector<double> v = scaled(*srcs[s], b);
                        for (long long q = 0; q < nimg; ++q) img[q] += v[q];
                    }
                    const char* stem[3] = {"direct_", "scatt_", "direc0_"};
                    ok = put(std::string(stem[s]) + chname[ich] + suf, {d.nyim, d.nxim}, img.data(), img.size(),
                             "surface brightness [erg/s/cm^2/sr]", kw);
                }
            }
        } else {
            for (int ch = 0; ch < d.nchan && ok; ++ch) {
                std::vector<double> v = scaled(dir, ch);
                ok = put(std::string("direct_") + chname[ch] + suf, {d.nyim, d.nxim}, v.data(), v.size(),
                         "direct surface brightness [erg/s/cm^2/sr]", kw);
                v = scaled(sca, ch);
                if (ok) ok = put(std::string("scatt_") + chname[ch] + suf, {d.nyim, d.nxim}, v.data(), v.size(),
                                 "scattered surface brightness [erg/s/cm^2/sr]", kw);
                if (ok && d.direc0) {
                    v = scaled(dir0, ch);
                    ok = put(std::string("direc0_") + chname[ch] + suf, {d.nyim, d.nxim}, v.data(), v.size(),
                             "unattenuated direct surface brightness [erg/s/cm^2/sr]", kw);
                }
            }
        }
    }
    if (!ok) {
        c->last_error = "mochii_write_image: cannot write into " + dir_name;
        return MOCHII_ERR_BAD_PARAM;
    }
    const std::string j = "{\n  \"format\": \"mochii peel-off images: one .npy per image block (FP64, C order; the "
                          "reference's image img(nxim, nyim) is shape (nyim, nxim))\",\n  \"nobs\": " +
                          std::to_string(d.nobs) + ",\n  \"datasets\": [\n" + entries + "\n  ]\n}\n";
    FILE* f = std::fopen((dir_name + "/header.json").c_str(), "w");
    if (!f || std::fwrite(j.data(), 1, j.size(), f) != j.size() || std::fclose(f) != 0) {
        c->last_error = "mochii_write_image: cannot write header.json";
        return MOCHII_ERR_BAD_PARAM;
    }
    return MOCHII_OK;
}
