// rms_io.cpp -- the reference simulator's run-directory text formats.
//
// Inputs are read with the same stream extraction the reference uses
// (hpc_code/lib/main.cu:414-482, main_PGSE.cu:440-506), so any file the
// reference accepts is read to the same numbers; unlike the reference, a
// missing or short file is an error instead of silent zeros.  Outputs are
// written with the reference's exact stream formatting (precision 15 for the
// result tables, the default 6 for sim_para.txt and diff_time.txt;
// main.cu:550-615, main_PGSE.cu:596-669), so analysis/readRMS.m and
// readRMS_pgse.m read them unchanged.
#include <sys/stat.h>

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "rms_sim.h"

namespace rms {
namespace {

std::string join(const char* dir, const char* name) {
    std::string p(dir ? dir : ".");
    if (!p.empty() && p.back() != '/') p += '/';
    return p + name;
}

bool exists(const std::string& p) {
    struct stat st;
    return ::stat(p.c_str(), &st) == 0;
}

// Read `n` values of type T from a text file with operator>> (the reference's reader).
template <class T>
int read_values(const std::string& path, size_t n, std::vector<T>& out, bool allow_more = true) {
    std::ifstream f(path);
    if (!f) return set_error(RMS_ERR_IO, "cannot open " + path);
    out.resize(n);
    for (size_t i = 0; i < n; ++i) {
        if (!(f >> out[i])) {
            std::ostringstream m;
            m << path << ": expected " << n << " values, read " << i;
            return set_error(RMS_ERR_FORMAT, m.str());
        }
    }
    if (!allow_more) {
        T extra;
        if (f >> extra) {
            std::ostringstream m;
            m << path << ": more than the " << n << " expected values";
            return set_error(RMS_ERR_FORMAT, m.str());
        }
    }
    return RMS_OK;
}

int count_values(const std::string& path, size_t& n) {
    std::ifstream f(path);
    if (!f) return set_error(RMS_ERR_IO, "cannot open " + path);
    std::string tok;
    n = 0;
    while (f >> tok) ++n;
    return RMS_OK;
}

}  // namespace

// fiber.txt: n unsigned integers separated by whitespace, k fastest
// (writer analysis/setupRMS.m:17-23, reader main.cu:461-466).  Hand-rolled
// because a 256x256x2048 lattice is 134 M numbers.
int parse_lattice_text(const std::string& path, size_t n, std::vector<uint8_t>& out, int nc) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return set_error(RMS_ERR_IO, "cannot open " + path);
    out.assign(n, 0);
    std::vector<char> buf(1 << 22);
    size_t count = 0;
    unsigned long cur = 0;
    bool in_num = false;
    int rc = RMS_OK;
    std::string bad;
    for (;;) {
        const size_t got = std::fread(buf.data(), 1, buf.size(), f);
        if (got == 0) break;
        for (size_t i = 0; i < got; ++i) {
            const char c = buf[i];
            if (c >= '0' && c <= '9') {
                cur = cur * 10 + (unsigned long)(c - '0');
                if (cur > 255) cur = 256;  // saturate; rejected below
                in_num = true;
            } else if (c == ' ' || c == '\n' || c == '\t' || c == '\r') {
                if (in_num) {
                    if (count < n) {
                        if (cur >= (unsigned long)nc) { rc = RMS_ERR_RANGE; bad = std::to_string(cur); }
                        out[count] = (uint8_t)(cur > 255 ? 255 : cur);
                    }
                    ++count;
                    cur = 0;
                    in_num = false;
                }
            } else {
                std::fclose(f);
                return set_error(RMS_ERR_FORMAT, path + ": unexpected character in lattice");
            }
        }
    }
    if (in_num) {
        if (count < n) {
            if (cur >= (unsigned long)nc) { rc = RMS_ERR_RANGE; bad = std::to_string(cur); }
            out[count] = (uint8_t)(cur > 255 ? 255 : cur);
        }
        ++count;
    }
    std::fclose(f);
    if (count < n) {
        std::ostringstream m;
        m << path << ": expected " << n << " labels, read " << count;
        return set_error(RMS_ERR_FORMAT, m.str());
    }
    if (rc != RMS_OK) return set_error(rc, path + ": label " + bad + " is not below Nc");
    return RMS_OK;
}

// fiber.bin (engine extension): the same labels as fiber.txt, one byte per
// voxel, i outer, k fastest, nothing else -- read as it lies instead of
// parsed (a 256x256x2048 lattice is 134 M integers of text).
int read_lattice_binary(const std::string& path, size_t n, std::vector<uint8_t>& out, int nc) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return set_error(RMS_ERR_IO, "cannot open " + path);
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size < 0 || (size_t)size != n) {
        std::fclose(f);
        std::ostringstream m;
        m << path << ": " << size << " bytes; the lattice has " << n << " voxels (one byte each)";
        return set_error(RMS_ERR_FORMAT, m.str());
    }
    out.assign(n, 0);
    const size_t got = std::fread(out.data(), 1, n, f);
    std::fclose(f);
    if (got != n) return set_error(RMS_ERR_IO, path + ": short read");
    for (size_t i = 0; i < n; ++i)
        if (out[i] >= nc) {
            std::ostringstream m;
            m << path << ": label " << (int)out[i] << " at voxel " << i << " is not below Nc";
            return set_error(RMS_ERR_RANGE, m.str());
        }
    return RMS_OK;
}

int load_run_dir(const char* dir, int mode, rms_sim* s) {
    const std::string grad_path = join(dir, "gradient_time.txt");
    if (mode == RMS_MODE_AUTO) mode = exists(grad_path) ? RMS_MODE_PGSE : RMS_MODE_NARROW;
    if (mode != RMS_MODE_NARROW && mode != RMS_MODE_PGSE)
        return set_error(RMS_ERR_ARG, "mode must be RMS_MODE_NARROW, RMS_MODE_PGSE or RMS_MODE_AUTO");
    s->mode = mode;

    // simParamInput.txt: dt TN NPar [Nbvec] Nc res NPix1 NPix2 NPix3
    // (main.cu:414-419; main_PGSE.cu:440-445 has no Nbvec)
    const std::string pp = join(dir, "simParamInput.txt");
    size_t nvals = 0;
    int rc = count_values(pp, nvals);
    if (rc) return rc;
    const size_t want = (mode == RMS_MODE_NARROW) ? 9 : 8;
    if (nvals != want) {
        std::ostringstream m;
        m << pp << ": " << nvals << " values; the "
          << (mode == RMS_MODE_NARROW ? "narrow-pulse layout (dt TN NPar Nbvec Nc res NPix1 NPix2 NPix3)"
                                      : "PGSE layout (dt TN NPar Nc res NPix1 NPix2 NPix3)")
          << " has " << want;
        return set_error(RMS_ERR_FORMAT, m.str());
    }
    {
        std::ifstream f(pp);
        int tn = 0, npar = 0, nbvec = 0, nc = 0;
        f >> s->dt >> tn >> npar;
        if (mode == RMS_MODE_NARROW) f >> nbvec;
        f >> nc >> s->res >> s->n1 >> s->n2 >> s->n3;
        if (!f) return set_error(RMS_ERR_FORMAT, pp + ": malformed");
        s->tn = tn;
        s->npar = npar;
        s->nc = nc;
        if (nc < 1 || nc > 255) return set_error(RMS_ERR_RANGE, pp + ": Nc out of range");
        if (nbvec < 0) return set_error(RMS_ERR_RANGE, pp + ": Nbvec < 0");
        if ((rc = read_values(join(dir, "diffusivity.txt"), (size_t)nc, s->diffusivity))) return rc;
        if ((rc = read_values(join(dir, "T2.txt"), (size_t)nc, s->t2))) return rc;
        if (mode == RMS_MODE_NARROW) {
            if ((rc = read_values(join(dir, "bval.txt"), (size_t)nbvec, s->bval))) return rc;
            if ((rc = read_values(join(dir, "bvec.txt"), (size_t)nbvec * 3, s->bvec))) return rc;
        } else {
            std::vector<int> ng;
            if ((rc = read_values(join(dir, "gradient_Ngrad.txt"), 1, ng))) return rc;
            if (ng[0] < 0) return set_error(RMS_ERR_RANGE, "gradient_Ngrad.txt: Ngrad < 0");
            if ((rc = read_values(grad_path, (size_t)ng[0] * 6, s->grad))) return rc;
        }
    }
    if ((rc = finalize_config(s))) return rc;
    const size_t nvox = (size_t)s->n1 * s->n2 * s->n3;
    const std::string bin = join(dir, "fiber.bin");
    if (exists(bin)) {
        if ((rc = read_lattice_binary(bin, nvox, s->labels, s->nc))) return rc;
    } else if ((rc = parse_lattice_text(join(dir, "fiber.txt"), nvox, s->labels, s->nc))) {
        return rc;
    }
    s->have_lattice = true;
    s->lattice_dirty = true;
    return RMS_OK;
}

int write_run_dir(const rms_sim* s, const char* dir) {
    if (!s->have_results) return set_error(RMS_ERR_STATE, "no results: run the simulation first");
    const int T = s->timepoints;
    const int nc = s->nc;
    auto open = [&](const char* name, std::ofstream& f) -> int {
        f.open(join(dir, name));
        if (!f) return set_error(RMS_ERR_IO, std::string("cannot write ") + join(dir, name));
        return RMS_OK;
    };
    int rc;
    std::ofstream fs0, fdx2, fdx4, fsig, fnp;
    if ((rc = open("sig0.txt", fs0)) || (rc = open("dx2.txt", fdx2)) || (rc = open("dx4.txt", fdx4)) ||
        (rc = open(s->mode == RMS_MODE_NARROW ? "sigRe.txt" : (s->mode == RMS_MODE_PGSE ? "sig.txt" : "sigw.txt"), fsig)) ||
        (rc = open("NPar_count.txt", fnp)))
        return rc;
    fs0.precision(15);
    fdx2.precision(15);
    fdx4.precision(15);
    fsig.precision(15);
    const int nb = s->nbvec();
    for (int i = 0; i < T; i++) {                      // main.cu:561-599
        fs0 << s->sig0[i] << std::endl;
        for (int j = 0; j < 6; j++) {
            if (j == 5) fdx2 << s->dx2[i * 6 + j] << std::endl;
            else fdx2 << s->dx2[i * 6 + j] << "\t";
        }
        for (int j = 0; j < 15; j++) {
            if (j == 14) fdx4 << s->dx4[i * 15 + j] << std::endl;
            else fdx4 << s->dx4[i * 15 + j] << "\t";
        }
        if (s->mode == RMS_MODE_NARROW) {
            for (int j = 0; j < nb; j++) {
                if (j == nb - 1) fsig << s->sigre[(size_t)i * nb + j] << std::endl;
                else fsig << s->sigre[(size_t)i * nb + j] << "\t";
            }
        }
        for (int j = 0; j < nc; j++) {
            if (j == nc - 1) fnp << s->npar_count[i * nc + j] << std::endl;
            else fnp << s->npar_count[i * nc + j] << "\t";
        }
    }
    if (s->mode == RMS_MODE_PGSE) {                    // main_PGSE.cu:649-651
        for (int i = 0; i < s->ngrad(); i++) fsig << s->sig[i] << std::endl;
    }
    if (s->mode == RMS_MODE_WAVEFORM) {                // extension: one row "cos<TAB>sin" per waveform
        for (int i = 0; i < s->nwave; i++) fsig << s->sigw[2 * i] << "\t" << s->sigw[2 * i + 1] << std::endl;
    }
    for (std::ofstream* f : {&fs0, &fdx2, &fdx4, &fsig, &fnp}) {
        f->close();
        if (f->fail()) return set_error(RMS_ERR_IO, std::string("write failed in ") + dir);
    }
    std::ofstream para;                                 // main.cu:606-609
    if ((rc = open("sim_para.txt", para))) return rc;
    para << s->dt << std::endl << s->tn << std::endl << s->npar << std::endl;
    para << s->res << std::endl;
    para.close();
    std::ofstream tdout;                                // main.cu:611-615
    if ((rc = open("diff_time.txt", tdout))) return rc;
    for (int i = 0; i < T; i++) tdout << s->td[i] << std::endl;
    tdout.close();
    if (para.fail() || tdout.fail()) return set_error(RMS_ERR_IO, std::string("write failed in ") + dir);
    return RMS_OK;
}

}  // namespace rms
