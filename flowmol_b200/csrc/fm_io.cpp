// fm_io.cpp -- Flowmol's restart file and keyword input, host side.
//
// final_state layout (parallel_io.MPI2.f90:1495-1726): a body of FP64
// records, one per molecule -- tag, r(3), v(3), [rtrue(3) if rtrue_flag],
// [rtether(3) if the tag is a tethered one], [moltype if mie_potential],
// [glob_no if global_numbering], [8 monomer values if potential_flag] --
// followed by a header appended at the end of the file: 18 int32 (globalnp,
// initialnunits(3), Nsteps or iter, tplot, seed(2), periodic(3),
// potential_flag, rtrue_flag, solvent_flag, nmonomers, npx, npy, npz),
// procnp(nproc), proctethernp(nproc), 14 FP64 (globaldomain(3), density,
// rcutoff, delta_t, elapsedtime, simtime, k_c, R_0, eps_pp, eps_ps, eps_ss,
// delta_rneighbr(1)), mie_potential, global_numbering (int32) and the int64
// byte offset at which the header starts.  Native byte order.
//
// Keyword input (setup_read_input.f90 with locate, functions_lib.f90:1139-1193):
// a keyword is found on the first line whose first token starts with it; its
// values are the first tokens of the following lines, one per read.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "fm_common.cuh"
#include "flowmol_b200.h"

namespace {

int iofail(int code, const std::string &m)
{
    fm::set_last_error(m.c_str());
    return code;
}

bool is_tether_tag(int t) { return t == 3 || t == 5 || t == 6 || t == 7 || t == 10; }

template <typename T>
bool get(const std::vector<char> &b, size_t &pos, T &out)
{
    if (pos + sizeof(T) > b.size()) return false;
    std::memcpy(&out, b.data() + pos, sizeof(T));
    pos += sizeof(T);
    return true;
}

template <typename T>
void put(std::vector<char> &b, const T &v)
{
    const char *p = reinterpret_cast<const char *>(&v);
    b.insert(b.end(), p, p + sizeof(T));
}

}  // namespace

extern "C" int fm_read_final_state(const char *path, fm_restart_header *h, int32_t cap, double *r, double *v,
                                   int32_t *tag, double *rtether, int32_t *glob_no, double *rtrue,
                                   int32_t *moltype, double *monomer)
{
    if (!path || !h) return iofail(FM_ERR_ARG, "null argument");
    std::ifstream f(path, std::ios::binary);
    if (!f) return iofail(FM_ERR_IO, std::string("cannot open ") + path);
    std::vector<char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    if (b.size() < 8) return iofail(FM_ERR_IO, "restart file too short");
    int64_t hp = 0;
    std::memcpy(&hp, b.data() + b.size() - 8, 8);
    if (hp < 0 || (size_t)hp > b.size() - 8) return iofail(FM_ERR_IO, "bad header offset");
    std::memset(h, 0, sizeof *h);
    size_t pos = (size_t)hp;
    int32_t ints[18];
    for (int k = 0; k < 18; k++)
        if (!get(b, pos, ints[k])) return iofail(FM_ERR_IO, "truncated header");
    h->globalnp = ints[0];
    for (int k = 0; k < 3; k++) h->initialnunits[k] = ints[1 + k];
    h->nsteps = ints[4];
    h->tplot = ints[5];
    h->seed[0] = ints[6]; h->seed[1] = ints[7];
    for (int k = 0; k < 3; k++) h->periodic[k] = ints[8 + k];
    h->potential_flag = ints[11]; h->rtrue_flag = ints[12]; h->solvent_flag = ints[13]; h->nmonomers = ints[14];
    h->npx = ints[15]; h->npy = ints[16]; h->npz = ints[17];
    long long nproc = (long long)h->npx * h->npy * h->npz;
    if (nproc <= 0 || nproc > FM_RESTART_MAXPROC) return iofail(FM_ERR_IO, "processor topology out of range");
    h->nproc = (int32_t)nproc;
    for (int p = 0; p < nproc; p++)
        if (!get(b, pos, h->procnp[p])) return iofail(FM_ERR_IO, "truncated header");
    for (int p = 0; p < nproc; p++)
        if (!get(b, pos, h->proctethernp[p])) return iofail(FM_ERR_IO, "truncated header");
    double dbl[14];
    for (int k = 0; k < 14; k++)
        if (!get(b, pos, dbl[k])) return iofail(FM_ERR_IO, "truncated header");
    for (int k = 0; k < 3; k++) h->globaldomain[k] = dbl[k];
    h->density = dbl[3]; h->rcutoff = dbl[4]; h->delta_t = dbl[5]; h->elapsedtime = dbl[6]; h->simtime = dbl[7];
    h->k_c = dbl[8]; h->R_0 = dbl[9]; h->eps_pp = dbl[10]; h->eps_ps = dbl[11]; h->eps_ss = dbl[12];
    h->delta_rneighbr = dbl[13];
    if (!get(b, pos, h->mie_potential) || !get(b, pos, h->global_numbering))
        return iofail(FM_ERR_IO, "truncated header");
    h->header_pos = hp;
    if (!r && !v) return FM_OK;  // header only
    const int n = h->globalnp;
    if (cap < n) return iofail(FM_ERR_ARG, "arrays smaller than globalnp");
    size_t q = 0;
    std::vector<char> body(b.begin(), b.begin() + hp);
    for (int i = 0; i < n; i++) {
        double t, x[3], u[3];
        if (!get(body, q, t)) return iofail(FM_ERR_IO, "truncated body");
        for (int k = 0; k < 3; k++)
            if (!get(body, q, x[k])) return iofail(FM_ERR_IO, "truncated body");
        for (int k = 0; k < 3; k++)
            if (!get(body, q, u[k])) return iofail(FM_ERR_IO, "truncated body");
        const int it = (int)t;
        if (tag) tag[i] = it;
        for (int k = 0; k < 3; k++) {
            if (r) r[3 * (size_t)i + k] = x[k];
            if (v) v[3 * (size_t)i + k] = u[k];
        }
        if (h->rtrue_flag == 1) {
            for (int k = 0; k < 3; k++) {
                double y;
                if (!get(body, q, y)) return iofail(FM_ERR_IO, "truncated body");
                if (rtrue) rtrue[3 * (size_t)i + k] = y;
            }
        }
        if (is_tether_tag(it)) {
            for (int k = 0; k < 3; k++) {
                double y;
                if (!get(body, q, y)) return iofail(FM_ERR_IO, "truncated body");
                if (rtether) rtether[3 * (size_t)i + k] = y;
            }
        } else if (rtether) {
            for (int k = 0; k < 3; k++) rtether[3 * (size_t)i + k] = 0.0;
        }
        if (h->mie_potential == 1) {
            double y;
            if (!get(body, q, y)) return iofail(FM_ERR_IO, "truncated body");
            if (moltype) moltype[i] = (int32_t)y;
        }
        if (h->global_numbering == 1) {
            double y;
            if (!get(body, q, y)) return iofail(FM_ERR_IO, "truncated body");
            if (glob_no) glob_no[i] = (int32_t)y;
        } else if (glob_no) {
            glob_no[i] = i + 1;
        }
        if (h->potential_flag == 1) {
            for (int k = 0; k < 8; k++) {
                double y;
                if (!get(body, q, y)) return iofail(FM_ERR_IO, "truncated body");
                if (monomer) monomer[8 * (size_t)i + k] = y;
            }
        }
    }
    if (q != body.size()) return iofail(FM_ERR_IO, "body size does not match the header flags");
    return FM_OK;
}

extern "C" int fm_write_final_state(const char *path, const fm_restart_header *h, const double *r, const double *v,
                                    const int32_t *tag, const double *rtether, const int32_t *glob_no,
                                    const double *rtrue, const int32_t *moltype, const double *monomer)
{
    if (!path || !h || !r || !v) return iofail(FM_ERR_ARG, "null argument");
    const long long nproc = (long long)h->npx * h->npy * h->npz;
    if (nproc <= 0 || nproc > FM_RESTART_MAXPROC) return iofail(FM_ERR_ARG, "processor topology out of range");
    std::vector<char> b;
    b.reserve((size_t)h->globalnp * 8 * 8 + 1024);
    for (int i = 0; i < h->globalnp; i++) {
        const int it = tag ? tag[i] : 0;
        put(b, (double)it);
        for (int k = 0; k < 3; k++) put(b, r[3 * (size_t)i + k]);
        for (int k = 0; k < 3; k++) put(b, v[3 * (size_t)i + k]);
        if (h->rtrue_flag == 1)
            for (int k = 0; k < 3; k++) put(b, rtrue ? rtrue[3 * (size_t)i + k] : 0.0);
        if (is_tether_tag(it))
            for (int k = 0; k < 3; k++) put(b, rtether ? rtether[3 * (size_t)i + k] : 0.0);
        if (h->mie_potential == 1) put(b, (double)(moltype ? moltype[i] : 0));
        if (h->global_numbering == 1) put(b, (double)(glob_no ? glob_no[i] : i + 1));
        if (h->potential_flag == 1)
            for (int k = 0; k < 8; k++) put(b, monomer ? monomer[8 * (size_t)i + k] : 0.0);
    }
    const int64_t hp = (int64_t)b.size();
    int32_t ints[18] = {h->globalnp, h->initialnunits[0], h->initialnunits[1], h->initialnunits[2], h->nsteps,
                        h->tplot, h->seed[0], h->seed[1], h->periodic[0], h->periodic[1], h->periodic[2],
                        h->potential_flag, h->rtrue_flag, h->solvent_flag, h->nmonomers, h->npx, h->npy, h->npz};
    for (int k = 0; k < 18; k++) put(b, ints[k]);
    for (int p = 0; p < nproc; p++) put(b, h->procnp[p]);
    for (int p = 0; p < nproc; p++) put(b, h->proctethernp[p]);
    const double dbl[14] = {h->globaldomain[0], h->globaldomain[1], h->globaldomain[2], h->density, h->rcutoff,
                            h->delta_t, h->elapsedtime, h->simtime, h->k_c, h->R_0, h->eps_pp, h->eps_ps,
                            h->eps_ss, h->delta_rneighbr};
    for (int k = 0; k < 14; k++) put(b, dbl[k]);
    put(b, h->mie_potential);
    put(b, h->global_numbering);
    put(b, hp);
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) return iofail(FM_ERR_IO, std::string("cannot create ") + path);
    f.write(b.data(), (std::streamsize)b.size());
    if (!f) return iofail(FM_ERR_IO, std::string("write failed: ") + path);
    return FM_OK;
}

// ---------------------------------------------------------------------------
// keyword input
// ---------------------------------------------------------------------------

namespace {

struct Deck {
    std::vector<std::string> lines;
    // first token of a line, Fortran list-directed style (blank/comma ends it)
    static std::string token(const std::string &s)
    {
        size_t a = s.find_first_not_of(" \t\r");
        if (a == std::string::npos) return "";
        size_t e = s.find_first_of(" \t\r,/", a);
        return s.substr(a, e == std::string::npos ? std::string::npos : e - a);
    }
    // index of the first line whose first token starts with the keyword
    long find(const std::string &key) const
    {
        for (size_t i = 0; i < lines.size(); i++) {
            std::string t = token(lines[i]);
            if (t.compare(0, key.size(), key) == 0 && t.size() >= key.size()) return (long)i;
        }
        return -1;
    }
    // next `count` values, one per following non-blank record
    bool values(long at, int count, std::vector<std::string> &out) const
    {
        out.clear();
        for (size_t i = (size_t)at + 1; i < lines.size() && (int)out.size() < count; i++) {
            std::string t = token(lines[i]);
            if (t.empty()) continue;
            out.push_back(t);
        }
        return (int)out.size() == count;
    }
};

bool to_double(std::string s, double &out)
{
    for (char &c : s)
        if (c == 'd' || c == 'D') c = 'e';
    char *end = nullptr;
    out = std::strtod(s.c_str(), &end);
    return end && *end == '\0' && end != s.c_str();
}

bool to_int(const std::string &s, int32_t &out)
{
    double d;
    if (!to_double(s, d) || d != std::floor(d)) return false;
    out = (int32_t)d;
    return true;
}

}  // namespace

extern "C" int fm_read_input(const char *path, fm_input *in)
{
    if (!path || !in) return iofail(FM_ERR_ARG, "null argument");
    std::ifstream f(path);
    if (!f) return iofail(FM_ERR_IO, std::string("cannot open ") + path);
    Deck deck;
    std::string line;
    while (std::getline(f, line)) deck.lines.push_back(line);
    std::memset(in, 0, sizeof *in);
    // defaults of the optional keywords (setup_read_input.f90)
    in->rebuild_criteria = 0;
    in->fixed_rebuild = 1;
    in->periodic[0] = in->periodic[1] = in->periodic[2] = 1;
    in->teth_k[0] = 0.0; in->teth_k[1] = 5000.0; in->teth_k[2] = 5000000.0;
    std::vector<std::string> vals;
    std::string missing;
    auto req_d = [&](const char *key, double *dst, int n) {
        long at = deck.find(key);
        if (at < 0 || !deck.values(at, n, vals)) { missing += std::string(key) + " "; return; }
        for (int k = 0; k < n; k++)
            if (!to_double(vals[(size_t)k], dst[k])) missing += std::string(key) + "(value) ";
    };
    auto req_i = [&](const char *key, int32_t *dst, int n) {
        long at = deck.find(key);
        if (at < 0 || !deck.values(at, n, vals)) { missing += std::string(key) + " "; return; }
        for (int k = 0; k < n; k++)
            if (!to_int(vals[(size_t)k], dst[k])) missing += std::string(key) + "(value) ";
    };
    auto opt_d = [&](const char *key, double *dst, int n) -> bool {
        long at = deck.find(key);
        if (at < 0 || !deck.values(at, n, vals)) return false;
        for (int k = 0; k < n; k++)
            if (!to_double(vals[(size_t)k], dst[k])) return false;
        return true;
    };
    auto opt_i = [&](const char *key, int32_t *dst, int n) -> bool {
        long at = deck.find(key);
        if (at < 0 || !deck.values(at, n, vals)) return false;
        for (int k = 0; k < n; k++)
            if (!to_int(vals[(size_t)k], dst[k])) return false;
        return true;
    };
    req_i("ENSEMBLE", &in->ensemble, 1);
    req_d("DENSITY", &in->density, 1);
    req_d("RCUTOFF", &in->rcutoff, 1);
    req_i("INITIALNUNITS", in->initialnunits, 3);
    req_d("INPUTTEMPERATURE", &in->inputtemperature, 1);
    req_i("INTEGRATION_ALGORITHM", &in->integration_algorithm, 1);
    req_i("FORCE_LIST", &in->force_list, 1);
    req_i("NSTEPS", &in->nsteps, 1);
    req_d("DELTA_T", &in->delta_t, 1);
    req_i("TPLOT", &in->tplot, 1);
    {  // DELTA_RNEIGHBR: one value, or three (setup_read_input.f90:759-779)
        long at = deck.find("DELTA_RNEIGHBR");
        double d[3];
        if (at < 0 || !deck.values(at, 1, vals) || !to_double(vals[0], d[0])) {
            missing += "DELTA_RNEIGHBR ";
        } else {
            d[1] = d[2] = d[0];
            std::vector<std::string> v3;
            if (deck.values(at, 3, v3) && to_double(v3[1], d[1]) && to_double(v3[2], d[2])) {
            } else {
                d[1] = d[2] = d[0];
            }
            for (int k = 0; k < 3; k++) in->delta_rneighbr[k] = d[k];
        }
    }
    if (!missing.empty()) return iofail(FM_ERR_IO, "required input missing or malformed: " + missing);
    int32_t rb;
    if (opt_i("REBUILD_CRITERIA", &rb, 1)) {
        in->rebuild_criteria = rb;
        if (rb == 1) {
            long at = deck.find("REBUILD_CRITERIA");
            if (deck.values(at, 2, vals)) to_int(vals[1], in->fixed_rebuild);
        }
    }
    opt_i("POTENTIAL_FLAG", &in->potential_flag, 1);
    opt_i("PERIODIC", in->periodic, 3);
    opt_i("GLOBAL_NUMBERING", &in->global_numbering, 1);
    {  // SORT_FLAG: sort_flag, sort_freq, sortblocksize (setup_read_input.f90:818-827)
        int32_t sf[3];
        if (opt_i("SORT_FLAG", sf, 3)) {
            in->sort_flag = sf[0];
            in->sort_freq = sf[1];
            in->sortblocksize = sf[2];
        }
    }
    opt_i("PRESSURE_OUTFLAG", &in->pressure_outflag, 1);
    opt_i("SLRC_FLAG", &in->sLRC_flag, 1);
    {
        int32_t mie[1];
        if (opt_i("MIE_POTENTIAL", mie, 1)) in->mie_potential = mie[0];
    }
    // INITIAL_CONFIG_FLAG 1 names a special case whose own block follows
    // (setup_read_input.f90:188-199); the polymer ones set potential_flag 1 and
    // the WCA cutoff (:232, 256)
    std::string special;
    {
        long at = deck.find("INITIAL_CONFIG_FLAG");
        int32_t icf = 0;
        if (at >= 0 && deck.values(at, 2, vals) && to_int(vals[0], icf) && icf == 1) special = vals[1];
    }
    if (special == "dense_fene") {  // DENSE_FENE: nmonomers, k_c, r_0, density, initialnunits(3) (:229-254)
        long at = deck.find("DENSE_FENE");
        if (at < 0 || !deck.values(at, 7, vals)) return iofail(FM_ERR_IO, "dense_fene needs the DENSE_FENE block");
        double dd;
        in->potential_flag = 1;
        to_int(vals[0], in->nmonomers);
        if (to_double(vals[1], dd)) in->k_c = dd;
        if (to_double(vals[2], dd)) in->R_0 = dd;
        if (to_double(vals[3], dd)) in->density = dd;
        for (int k = 0; k < 3; k++) to_int(vals[(size_t)(4 + k)], in->initialnunits[k]);
        in->rcutoff = std::pow(2.0, 1.0 / 6.0);
    }
    if (special == "fene_solution" || special == "single_fene") {
        // FENE_SOLUTION: nmonomers, k_c, r_0, density, targetconc (:253-273)
        long at = deck.find("FENE_SOLUTION");
        if (at < 0 || !deck.values(at, 5, vals))
            return iofail(FM_ERR_IO, special + " needs the FENE_SOLUTION block");
        double dd;
        in->potential_flag = 1;
        to_int(vals[0], in->nmonomers);
        if (to_double(vals[1], dd)) in->k_c = dd;
        if (to_double(vals[2], dd)) in->R_0 = dd;
        if (to_double(vals[3], dd)) in->density = dd;
        if (to_double(vals[4], dd)) in->targetconc = dd;
        in->rcutoff = std::pow(2.0, 1.0 / 6.0);
        // SOLVENT_INFO: flag, then eps_pp, eps_ps, eps_ss when it is 1 (:275-296)
        at = deck.find("SOLVENT_INFO");
        if (at < 0 || !deck.values(at, 1, vals) || !to_int(vals[0], in->solvent_flag))
            return iofail(FM_ERR_IO, special + " needs the SOLVENT_INFO block");
        if (in->solvent_flag == 1) {
            if (!deck.values(at, 4, vals) || !to_double(vals[1], in->eps_pp) || !to_double(vals[2], in->eps_ps) ||
                !to_double(vals[3], in->eps_ss))
                return iofail(FM_ERR_IO, "SOLVENT_INFO 1 needs eps_pp, eps_ps and eps_ss");
        } else if (in->solvent_flag != 0) {
            return iofail(FM_ERR_IO, "Unrecognised solvent flag!");  // :293
        }
    }
    opt_d("TETHEREDDISTTOP", in->tethereddisttop, 3);
    opt_d("TETHEREDDISTBOTTOM", in->tethereddistbottom, 3);
    opt_d("THERMSTATTOP", in->thermstattop, 3);
    opt_d("THERMSTATBOTTOM", in->thermstatbottom, 3);
    opt_d("SLIDEDISTTOP", in->slidedisttop, 3);
    opt_d("SLIDEDISTBOTTOM", in->slidedistbottom, 3);
    opt_d("FIXDISTTOP", in->fixdisttop, 3);
    opt_d("FIXDISTBOTTOM", in->fixdistbottom, 3);
    opt_d("WALLSLIDEV", in->wallslidev, 3);
    opt_d("TETHERCOEFFICIENTS", in->teth_k, 3);
    in->thermostattemperature[0] = in->thermostattemperature[1] = in->inputtemperature;
    in->nthermo = 1;
    {  // THERMOSTATTEMPERATURE: as many values as parse, one region each (:127-146)
        long at = deck.find("THERMOSTATTEMPERATURE");
        if (at >= 0) {
            int cnt = 0;
            for (size_t i = (size_t)at + 1; i < deck.lines.size() && cnt < 2; i++) {
                std::string t = Deck::token(deck.lines[i]);
                double dd;
                if (t.empty()) continue;
                if (!to_double(t, dd)) break;
                in->thermostattemperature[cnt++] = dd;
            }
            if (cnt == 1) in->thermostattemperature[1] = in->thermostattemperature[0];
            if (cnt > 0) in->nthermo = cnt;
        }
    }
    // GLOBAL_NUMBERING (setup_read_input.f90:835-847): polymers number their
    // beads in the monomer data instead, and numbering cannot sort
    if (in->potential_flag == 1) in->global_numbering = 0;
    if (in->global_numbering == 1 && in->sort_flag != 0)
        return iofail(FM_ERR_ARG, "Global number does not work with sort flag on");
    return FM_OK;
}
