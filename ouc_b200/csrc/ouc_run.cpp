// ouc_run: the reference's main() workflow as a command-line program over
// libouc.so -- build the model, migrate every shot, write each shot's
// Laplacian images and the stacks as raw float32 files with the reference's
// names, so that tools reading the reference's output read these unchanged.
//
// Reference workflow (P-S-seperating.cu, "PS:n"):
//   * sizes PS:14-26: Xn = Zn = 600, L = 200, N = 6, NT = 6000, FM = 30,
//     R = 1e-3, 40 shots; spacing PS:1685-1688: dt = 1 ms, dx = dz = 10 m;
//   * model PS:1999-2040: Vp 3400 / 3800 / 4500 m/s with boundaries at
//     interior depth 50 and 100 cells, Vs 2900 / 3800 m/s split at 100;
//   * geometry PS:2113-2114: source l at interior (5 l, 0), receivers on
//     interior row 0; records self-modelled and direct-wave muted;
//   * per-shot files PS:2379-2400: <out>/image_PP_lap_<nx>_<nz>_<l>.dat and
//     image_PS_lap_..., float32, interior nx x nz, x-major (z fastest);
//   * stack PS:2403-2467: the per-shot files read back in shot order and
//     summed in float32 into <out>/All_image_PP_lap.dat, All_image_PS_lap.dat.
// These are the defaults; every value can be overridden on the command line.
//
// Additions without a reference counterpart:
//   * <out>/All_image_{PP,PS}_lap_f64.dat and All_illum_f64.dat: the same
//     stack summed in float64 (illumination from the library's stack);
//   * <out>/manifest.txt: the run's parameters on its first line, then one
//     line "done <part> <l> <l> ..." per batch whose files are all complete
//     (each file is written under a temporary name and renamed, the line
//     with one append after them); <part> names the batch's FP64
//     illumination file.  --resume checks the parameters and skips the
//     shots of every line whose files are all present, so an interrupted
//     survey continues where it stopped; the stacks are always rebuilt from
//     the per-shot files and the listed illumination parts, so they do not
//     depend on how often the run was interrupted;
//   * --vp/--vs: the interior model from raw float32 files, x-major;
//     --true-vp/--true-vs: a second model to model the records with (the
//     migration then runs on --vp/--vs), otherwise records are self-modelled;
//   * --write-records: each shot's records as record_v{x,z}_<l>.dat
//     (float32, X x nt receiver-major as the reference keeps them in memory);
//   * --stop-after K: stop once K or more shots are done (whole batches), as
//     an interrupted run would; for testing the resume path.
//
// Exit status: 0 done, 1 usage or input error, 2 library error, 3 stopped
// early by --stop-after.
#include <sys/stat.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ouc.h"

namespace {

struct Run {
    int nx = 200, nz = 200, npml = 200, order = 6, nt = 6000;
    float dx = 10.f, dz = 10.f, dt = 1e-3f, fm = 30.f;
    double pml_r = 1e-3;
    int shots = 40, sx0 = 0, dsx = 5, sz = 0, rz = 0, mute = 1;
    int batch = 8, device = 0, stop_after = -1;
    int strip_level = OUC_STRIP_REFERENCE, image_align = OUC_IMAGE_REFERENCE;
    bool resume = false, write_records = false;
    std::string out = "image2", vp, vs, true_vp, true_vs;

    // the parameters a resumed run must share with the run it continues
    std::string signature() const {
        std::ostringstream s;
        s << "ouc_run nx=" << nx << " nz=" << nz << " npml=" << npml << " order=" << order << " nt=" << nt
          << " dx=" << dx << " dz=" << dz << " dt=" << dt << " fm=" << fm << " pml_r=" << pml_r << " shots=" << shots
          << " sx0=" << sx0 << " dsx=" << dsx << " sz=" << sz << " rz=" << rz << " mute=" << mute
          << " strip_level=" << strip_level << " image_align=" << image_align << " vp=" << (vp.empty() ? "reference" : vp)
          << " vs=" << (vs.empty() ? "reference" : vs) << " true_vp=" << true_vp << " true_vs=" << true_vs;
        return s.str();
    }
};

void usage() {
    std::printf(
        "usage: ouc_run [options]   (defaults: the reference's main(), P-S-seperating.cu)\n"
        "  --nx N --nz N --npml N --order N(2,5,6) --nt N --dx M --dz M --dt S --fm HZ --pml-r R\n"
        "  --shots N --sx0 I --dsx I --sz I --rz I --no-mute      geometry, interior cells\n"
        "  --vp FILE --vs FILE            interior model, float32 nx*nz x-major (default: built-in layers)\n"
        "  --true-vp FILE --true-vs FILE  model the records with this model instead\n"
        "  --strip-level reference|exact --image-align reference|exact\n"
        "  --batch N --device I --out DIR --resume --write-records --stop-after K\n");
}

bool read_floats(const std::string& path, std::vector<float>& v, size_t n) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    v.resize(n);
    const size_t got = std::fread(v.data(), sizeof(float), n, f);
    const bool extra = std::fgetc(f) != EOF;
    std::fclose(f);
    return got == n && !extra;
}

// Write under a temporary name, then rename: a file that exists under its
// final name is complete.
bool write_floats(const std::string& path, const float* p, size_t n) {
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(p, sizeof(float), n, f) == n;
    if (std::fclose(f) != 0 || !ok) return false;
    return std::rename(tmp.c_str(), path.c_str()) == 0;
}

bool write_doubles(const std::string& path, const double* p, size_t n) {
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(p, sizeof(double), n, f) == n;
    if (std::fclose(f) != 0 || !ok) return false;
    return std::rename(tmp.c_str(), path.c_str()) == 0;
}

long file_size(const std::string& path) {
    struct stat st;
    return stat(path.c_str(), &st) == 0 ? (long)st.st_size : -1;
}

std::string shot_file(const Run& r, const char* kind, int l) {
    return r.out + "/image_" + kind + "_lap_" + std::to_string(r.nx) + "_" + std::to_string(r.nz) + "_" +
           std::to_string(l) + ".dat";
}

// The reference's built-in model on the interior grid (PS:1999-2040).
void reference_model(const Run& r, std::vector<float>& vp, std::vector<float>& vs) {
    vp.assign((size_t)r.nx * r.nz, 0.f);
    vs.assign((size_t)r.nx * r.nz, 0.f);
    for (int i = 0; i < r.nx; ++i)
        for (int j = 0; j < r.nz; ++j) {
            vp[(size_t)i * r.nz + j] = j < 50 ? 3400.f : (j < 100 ? 3800.f : 4500.f);
            vs[(size_t)i * r.nz + j] = j < 100 ? 2900.f : 3800.f;
        }
}

bool parse(int argc, char** argv, Run& r) {
    for (int k = 1; k < argc; ++k) {
        const std::string a = argv[k];
        auto val = [&](void) -> const char* {
            if (k + 1 >= argc) {
                std::fprintf(stderr, "ouc_run: %s needs a value\n", a.c_str());
                return nullptr;
            }
            return argv[++k];
        };
        auto num_i = [&](int& dst) { const char* v = val(); if (!v) return false; char* e; dst = (int)std::strtol(v, &e, 10); return *e == 0; };
        auto num_f = [&](float& dst) { const char* v = val(); if (!v) return false; char* e; dst = std::strtof(v, &e); return *e == 0; };
        auto num_d = [&](double& dst) { const char* v = val(); if (!v) return false; char* e; dst = std::strtod(v, &e); return *e == 0; };
        auto str = [&](std::string& dst) { const char* v = val(); if (!v) return false; dst = v; return true; };
        auto mode = [&](int& dst) {
            const char* v = val();
            if (!v) return false;
            if (!std::strcmp(v, "reference")) dst = 0; else if (!std::strcmp(v, "exact")) dst = 1; else return false;
            return true;
        };
        bool ok = true;
        if (a == "--help" || a == "-h") { usage(); std::exit(0); }
        else if (a == "--nx") ok = num_i(r.nx);
        else if (a == "--nz") ok = num_i(r.nz);
        else if (a == "--npml") ok = num_i(r.npml);
        else if (a == "--order") ok = num_i(r.order);
        else if (a == "--nt") ok = num_i(r.nt);
        else if (a == "--dx") ok = num_f(r.dx);
        else if (a == "--dz") ok = num_f(r.dz);
        else if (a == "--dt") ok = num_f(r.dt);
        else if (a == "--fm") ok = num_f(r.fm);
        else if (a == "--pml-r") ok = num_d(r.pml_r);
        else if (a == "--shots") ok = num_i(r.shots);
        else if (a == "--sx0") ok = num_i(r.sx0);
        else if (a == "--dsx") ok = num_i(r.dsx);
        else if (a == "--sz") ok = num_i(r.sz);
        else if (a == "--rz") ok = num_i(r.rz);
        else if (a == "--no-mute") r.mute = 0;
        else if (a == "--vp") ok = str(r.vp);
        else if (a == "--vs") ok = str(r.vs);
        else if (a == "--true-vp") ok = str(r.true_vp);
        else if (a == "--true-vs") ok = str(r.true_vs);
        else if (a == "--strip-level") ok = mode(r.strip_level);
        else if (a == "--image-align") ok = mode(r.image_align);
        else if (a == "--batch") ok = num_i(r.batch);
        else if (a == "--device") ok = num_i(r.device);
        else if (a == "--out") ok = str(r.out);
        else if (a == "--resume") r.resume = true;
        else if (a == "--write-records") r.write_records = true;
        else if (a == "--stop-after") ok = num_i(r.stop_after);
        else { std::fprintf(stderr, "ouc_run: unknown option %s\n", a.c_str()); return false; }
        if (!ok) { std::fprintf(stderr, "ouc_run: bad value for %s\n", a.c_str()); return false; }
    }
    if (r.vp.empty() != r.vs.empty() || r.true_vp.empty() != r.true_vs.empty()) {
        std::fprintf(stderr, "ouc_run: give both --vp/--vs (and both --true-vp/--true-vs) or neither\n");
        return false;
    }
    if (r.shots < 1 || r.batch < 1 || r.nx < 1 || r.nz < 1 || r.nt < 2) {
        std::fprintf(stderr, "ouc_run: sizes, shots and batch must be positive\n");
        return false;
    }
    return true;
}

int lib_fail(ouc_ctx* ctx, int rc, const char* what) {
    std::fprintf(stderr, "ouc_run: %s: %s%s%s\n", what, ouc_strerror(rc), ctx ? ": " : "", ctx ? ouc_last_error(ctx) : "");
    return 2;
}

}  // namespace

int main(int argc, char** argv) {
    Run r;
    if (!parse(argc, argv, r)) { usage(); return 1; }
    mkdir(r.out.c_str(), 0755);
    const std::string manifest = r.out + "/manifest.txt";
    const size_t ni = (size_t)r.nx * r.nz;

    // shots already done (resume): lines "done <part> <l> ..." whose files are all there
    std::set<int> done;
    std::vector<std::string> lines;   // manifest lines kept
    std::vector<std::string> parts;   // their illumination parts
    if (r.resume) {
        std::ifstream in(manifest);
        std::string line;
        if (in && std::getline(in, line)) {
            if (line != r.signature()) {
                std::fprintf(stderr, "ouc_run: %s was written by a run with other parameters:\n  %s\n", manifest.c_str(),
                             line.c_str());
                return 1;
            }
            while (std::getline(in, line)) {
                std::istringstream ls(line);
                std::string word, part;
                if (!(ls >> word >> part) || word != "done") continue;
                bool ok = file_size(r.out + "/" + part) == (long)(ni * 8);
                std::vector<int> batch;
                int l;
                while (ls >> l) {
                    ok = ok && l >= 0 && l < r.shots && !done.count(l) &&
                         file_size(shot_file(r, "PP", l)) == (long)(ni * 4) &&
                         file_size(shot_file(r, "PS", l)) == (long)(ni * 4);
                    batch.push_back(l);
                }
                if (!ok || batch.empty()) continue;
                done.insert(batch.begin(), batch.end());
                lines.push_back(line);
                parts.push_back(part);
            }
        }
    }
    {   // (re)write the manifest: the signature and the lines kept
        std::ofstream m(manifest + ".tmp");
        m << r.signature() << "\n";
        for (const std::string& l : lines) m << l << "\n";
        m.close();
        if (!m || std::rename((manifest + ".tmp").c_str(), manifest.c_str()) != 0) {
            std::fprintf(stderr, "ouc_run: cannot write %s\n", manifest.c_str());
            return 1;
        }
    }

    std::vector<float> vp, vs, tvp, tvs;
    if (r.vp.empty()) {
        reference_model(r, vp, vs);
    } else if (!read_floats(r.vp, vp, ni) || !read_floats(r.vs, vs, ni)) {
        std::fprintf(stderr, "ouc_run: %s / %s must hold %zu float32 values each\n", r.vp.c_str(), r.vs.c_str(), ni);
        return 1;
    }
    if (!r.true_vp.empty() && (!read_floats(r.true_vp, tvp, ni) || !read_floats(r.true_vs, tvs, ni))) {
        std::fprintf(stderr, "ouc_run: %s / %s must hold %zu float32 values each\n", r.true_vp.c_str(),
                     r.true_vs.c_str(), ni);
        return 1;
    }

    ouc_config cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.nx = r.nx; cfg.nz = r.nz; cfg.npml = r.npml; cfg.half_order = r.order;
    cfg.dx = r.dx; cfg.dz = r.dz; cfg.dt = r.dt; cfg.nt = r.nt; cfg.pml_r = r.pml_r;
    cfg.model_layout = OUC_MODEL_INTERIOR;
    cfg.strip_level = r.strip_level;
    cfg.image_align = r.image_align;
    cfg.gather_layout = OUC_GATHER_XT;
    cfg.device = r.device;
    cfg.max_batch = r.batch;
    cfg.use_graphs = 1;

    std::vector<float> wavelet(r.nt);
    int t0 = 0;
    int rc = ouc_ricker(r.fm, r.dt, r.nt, wavelet.data(), &t0);   // PS:1954-1958
    if (rc) return lib_fail(nullptr, rc, "ouc_ricker");

    std::vector<ouc_shot> todo;
    std::vector<int> todo_l;
    for (int l = 0; l < r.shots; ++l) {
        if (done.count(l)) continue;
        ouc_shot s;
        s.sx = r.sx0 + l * r.dsx; s.sz = r.sz; s.rz = r.rz;
        s.src_type = OUC_SRC_THETA; s.t0 = t0; s.mute = r.mute;
        todo.push_back(s);
        todo_l.push_back(l);
    }
    std::printf("ouc_run: %d shots, %zu done before, %zu to migrate -> %s\n", r.shots, done.size(), todo.size(),
                r.out.c_str());

    if (!todo.empty()) {
        ouc_ctx* mig = nullptr;
        ouc_ctx* truth = nullptr;
        if ((rc = ouc_create(&cfg, vp.data(), vs.data(), nullptr, &mig))) return lib_fail(mig, rc, "ouc_create");
        if (!tvp.empty() && (rc = ouc_create(&cfg, tvp.data(), tvs.data(), nullptr, &truth))) {
            lib_fail(truth, rc, "ouc_create (record model)");
            ouc_destroy(mig);
            return 2;
        }
        int X = 0, Z = 0;
        ouc_dims(mig, &X, &Z);
        const size_t ng = (size_t)X * r.nt;
        std::vector<float> img((size_t)2 * r.batch * ni), recs;
        std::vector<double> il(ni);
        int migrated = 0, status = 0;
        for (size_t s0 = 0; s0 < todo.size() && status == 0; s0 += r.batch) {
            const int n = (int)std::min<size_t>(r.batch, todo.size() - s0);
            std::vector<float*> pp(n), ps(n);
            std::vector<const float*> rx, rz;
            for (int b = 0; b < n; ++b) {
                pp[b] = img.data() + (size_t)(2 * b) * ni;
                ps[b] = img.data() + (size_t)(2 * b + 1) * ni;
            }
            if (truth || r.write_records) {   // records modelled here (with the record model, if any)
                recs.assign((size_t)2 * n * ng, 0.f);
                ouc_ctx* rec_ctx = truth ? truth : mig;
                for (int b = 0; b < n && status == 0; ++b) {
                    float* gx = recs.data() + (size_t)(2 * b) * ng;
                    float* gz = recs.data() + (size_t)(2 * b + 1) * ng;
                    if ((rc = ouc_forward(rec_ctx, &todo[s0 + b], wavelet.data(), gx, gz, nullptr))) {
                        status = lib_fail(rec_ctx, rc, "ouc_forward");
                        break;
                    }
                    rx.push_back(gx);
                    rz.push_back(gz);
                    const std::string l = std::to_string(todo_l[s0 + b]);
                    if (r.write_records && (!write_floats(r.out + "/record_vx_" + l + ".dat", gx, ng) ||
                                            !write_floats(r.out + "/record_vz_" + l + ".dat", gz, ng))) {
                        std::fprintf(stderr, "ouc_run: cannot write the records of shot %s\n", l.c_str());
                        status = 1;
                    }
                }
                if (status) break;
            }
            // without a record model the library models each shot's records itself
            rc = ouc_rtm_batch(mig, n, &todo[s0], wavelet.data(), truth ? rx.data() : nullptr,
                               truth ? rz.data() : nullptr, pp.data(), ps.data());
            if (rc) { status = lib_fail(mig, rc, "ouc_rtm_batch"); break; }
            // the batch's FP64 illumination (the library's stack, cleared on reading), its
            // images, then one manifest line naming them all
            if ((rc = ouc_stack(mig, nullptr, nullptr, il.data(), 1))) { status = lib_fail(mig, rc, "ouc_stack"); break; }
            std::string part;
            for (int k = 0;; ++k) {
                part = "illum_" + std::to_string(todo_l[s0]) + "_" + std::to_string(k) + ".f64";
                if (file_size(r.out + "/" + part) < 0) break;
            }
            bool ok = write_doubles(r.out + "/" + part, il.data(), ni);
            std::string line = "done " + part;
            for (int b = 0; b < n && ok; ++b) {
                const int l = todo_l[s0 + b];
                ok = write_floats(shot_file(r, "PP", l), pp[b], ni) && write_floats(shot_file(r, "PS", l), ps[b], ni);
                line += " " + std::to_string(l);
            }
            if (ok) {
                std::ofstream m(manifest, std::ios::app);
                m << line << "\n";
                m.close();
                ok = (bool)m;
            }
            if (!ok) {
                std::fprintf(stderr, "ouc_run: cannot write the files of a batch in %s: %s\n", r.out.c_str(),
                             std::strerror(errno));
                status = 1;
                break;
            }
            parts.push_back(part);
            migrated += n;
            if (r.stop_after >= 0 && migrated >= r.stop_after) status = 3;
        }
        ouc_destroy(mig);
        if (truth) ouc_destroy(truth);
        if (status == 3) {
            std::printf("ouc_run: stopped after %d shots (--stop-after); rerun with --resume\n", migrated);
            return 3;
        }
        if (status) return status;
    }

    // stacks from the per-shot files, in shot order (PS:2403-2467), and the illumination parts
    std::vector<float> all_pp(ni, 0.f), all_ps(ni, 0.f), buf;
    std::vector<double> pp64(ni, 0.0), ps64(ni, 0.0), il64(ni, 0.0), part64(ni);
    for (int l = 0; l < r.shots; ++l) {
        if (!read_floats(shot_file(r, "PP", l), buf, ni)) { std::fprintf(stderr, "ouc_run: shot %d PP missing\n", l); return 1; }
        for (size_t k = 0; k < ni; ++k) { all_pp[k] += buf[k]; pp64[k] += buf[k]; }
        if (!read_floats(shot_file(r, "PS", l), buf, ni)) { std::fprintf(stderr, "ouc_run: shot %d PS missing\n", l); return 1; }
        for (size_t k = 0; k < ni; ++k) { all_ps[k] += buf[k]; ps64[k] += buf[k]; }
    }
    for (const std::string& part : parts) {
        FILE* fp = std::fopen((r.out + "/" + part).c_str(), "rb");
        const bool ok = fp && std::fread(part64.data(), sizeof(double), ni, fp) == ni;
        if (fp) std::fclose(fp);
        if (!ok) { std::fprintf(stderr, "ouc_run: %s/%s is short\n", r.out.c_str(), part.c_str()); return 1; }
        for (size_t q = 0; q < ni; ++q) il64[q] += part64[q];
    }
    if (!write_floats(r.out + "/All_image_PP_lap.dat", all_pp.data(), ni) ||
        !write_floats(r.out + "/All_image_PS_lap.dat", all_ps.data(), ni) ||
        !write_doubles(r.out + "/All_image_PP_lap_f64.dat", pp64.data(), ni) ||
        !write_doubles(r.out + "/All_image_PS_lap_f64.dat", ps64.data(), ni) ||
        !write_doubles(r.out + "/All_illum_f64.dat", il64.data(), ni)) {
        std::fprintf(stderr, "ouc_run: cannot write the stacks in %s\n", r.out.c_str());
        return 1;
    }
    std::printf("ouc_run: stacks written to %s\n", r.out.c_str());
    return 0;
}
