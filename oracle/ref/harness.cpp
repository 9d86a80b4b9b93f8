/*
 * Reference-oracle driver (test infrastructure only).
 *
 * Links the UNMODIFIED reference MAPP objects (compiled in place from the
 * reference tree by oracle/ref/Makefile against the single-rank mpi.h stub) and
 * drives the hot path exactly as the reference's own callers do, so the
 * outputs are the reference's results on our generated fixtures:
 *
 *   setup   = Min_LBFGS::init call order (min_l-bfgs.cpp:101-181):
 *             VecLst(x, c|type, id, f) + add_update(0) + reset_comm,
 *             forcefield->init(), atoms->ph_setup(1,..), neighbor->init(),
 *             neighbor->create_list(0,1), atoms->store_0()
 *   setx    = LineSearch::energy (line_search.cpp:180-195): write x, then
 *             atoms->update_0(0,1,..) (skin check, ghost refresh or rebuild)
 *   force / energy / crd / cdot / calcg call the ForceField virtuals.
 *   lbfgs   = Min_LBFGS (min_l-bfgs.cpp) constructed, init, run, fin, with
 *             the energy of every force_calc logged by the oracle subclass.
 *   cg      = Min_CG (min_cg.cpp), the same way.
 *   writecfg = WriteCFG (write_cfg.cpp) "write cfg 1 prefix x [c]" and one
 *             write_file(step) of the current state.
 *   adams   = Clock_Adams (clock_adams.cpp) constructed, init, run, then the
 *             owned c and the number of calc_g calls written before fin.
 *   bdf     = Clock_BDF (clock_bdf.cpp) the same way, plus the final time.
 *   md      = MD_NH "nvt" (md_nh.cpp) constructed, time_step / boltzmann set,
 *             init, run, then the owned x and x_d and one force_calc(1) at
 *             the final state written before fin.  Velocities are either
 *             given (x_d added and filled, then rescaled by init_vel) or made
 *             by create_vel.  x_0 is zeroed first: MD_NH::init never calls
 *             Atoms::store_0, so the reader's never-written x_0 would
 *             otherwise decide whether the first step rebuilds.
 *
 * Two harness-side measures (no change to reference arithmetic):
 *   - OracleDMD<Base>::coef restates ff_dmd_I.cpp:735-796 but routes "FS" to
 *     the class's own set_fs (ff_dmd_I.cpp:1300), because the stock DMD_I and
 *     DMD styles route "FS" to set_funcfl and crash for two species.
 *     (DMD_II already routes FS to set_fs, ff_dmd_II.cpp:757; its coef is used
 *     as is.)
 *   - OracleDMD<Base>::force_calc zeroes the per-pair scratch before calling
 *     the reference force_calc, because ff_dmd_I.cpp:120-144 zeroes it only on
 *     (re)allocation and pairs skipped by the cut / alpha tests would otherwise
 *     carry values from an earlier call into pass 2 (ff_dmd_I.cpp:376-383).
 *
 * Usage: mapp_ref_harness <command-file>
 * Each line of the command file is one operation (see run_command below).
 * Arrays are written as raw little-endian binaries next to a text meta file.
 */
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <sstream>
#include <fstream>

#include "MAPP.h"
#include "atoms.h"
#include "atom_types.h"
#include "neighbor.h"
#include "ff.h"
#include "ff_dmd_I.h"
#include "ff_dmd_II.h"
#include "ff_dmd.h"
#include "min_l-bfgs.h"
#include "min_cg.h"
#include "md_nh.h"
#include "clock_adams.h"
#include "clock_bdf.h"
#include "write_cfg.h"

using namespace MAPP_NS;

namespace {

/* eam_mode value of the reference's FINNIS_FL (ff_dmd_I.cpp:6) */
const int kFinnisFL = 3;

template <class Base>
class OracleDMD : public Base {
public:
    explicit OracleDMD(MAPP* m, bool route_fs) : Base(m), route_fs_(route_fs) {}

    void coef(int narg, char** arg) override
    {
        if (!route_fs_ || narg < 8 || strcmp(arg[6], "FS") != 0) {
            Base::coef(narg, arg);
            return;
        }
        /* restates ff_dmd_I.cpp:735-796 with FS routed to set_fs */
        double kb = 8.617332478e-5, hbar = 6.5821192815e-16;
        this->rsq_crd = atof(arg[1]);
        this->rsq_crd *= this->rsq_crd;
        this->set_weight_abs(atoi(arg[2]));
        this->alpha_min = atof(arg[3]);
        this->alpha_max = atof(arg[4]);
        double T = atof(arg[5]);
        this->clean_up();
        this->eam_mode = kFinnisFL;
        this->set_fs(narg - 7, &arg[7]);
        this->set_arrays();
        int nt = this->atom_types->no_types;
        for (int i = 0; i < nt; i++) {
            double mass = this->atom_types->mass[i];
            mass *= 1.0364269184093291236e-28;
            double deb_l = hbar * hbar * 2.0 / (mass * kb * T);
            this->c_0[i] = 1.5 * kb * T * (log(deb_l) - 1.0);
        }
        this->kbT = kb * T;
        this->beta = 1.0 / this->kbT;
        this->rc = (static_cast<double>(this->nr) - 1.0) * this->dr;
        this->rho_max = (static_cast<double>(this->nrho) - 1.0) * this->drho;
        this->cut_sq = this->rc * this->rc;
        this->mod_rc = this->rc + this->xi[this->no_i - 1] / sqrt(this->alpha_min);
        this->cut_sq_mod = this->mod_rc * this->mod_rc;
    }

    void force_calc(int st_clc, double* en_st) override
    {
        int nt = this->atom_types->no_types;
        if (this->max_pairs) {
            size_t n0 = (size_t)this->max_pairs * nt * nt;
            size_t n1 = (size_t)this->max_pairs * nt * (nt + 1) / 2;
            memset(this->rho, 0, n0 * sizeof(double));
            memset(this->drho_dr, 0, n0 * sizeof(double));
            memset(this->drho_dalpha, 0, n0 * sizeof(double));
            memset(this->phi, 0, n1 * sizeof(double));
            memset(this->dphi_dr, 0, n1 * sizeof(double));
            memset(this->dphi_dalpha, 0, n1 * sizeof(double));
        }
        Base::force_calc(st_clc, en_st);
        if (force_log) force_log->push_back(en_st[0]);
    }

    double energy_calc() override
    {
        n_energy++;
        return Base::energy_calc();
    }

    double calc_g(int chk, double alpha, double* a, double* g) override
    {
        n_calc_g++;
        return Base::calc_g(chk, alpha, a, g);
    }

    std::vector<double>* force_log = nullptr;  // en_st[0] of every force_calc while set
    long n_energy = 0;
    long n_calc_g = 0;

private:
    bool route_fs_;
};

/* the reference minimiser with its protected result fields exposed */
struct LbfgsRun : public Min_LBFGS {
    LbfgsRun(MAPP* m, int narg, char** arg) : Min_LBFGS(m, narg, arg) {}
    int code() const { return err; }
    double energy() const { return curr_energy; }
};

/* the reference CG minimiser with its protected result fields exposed */
struct CgRun : public Min_CG {
    CgRun(MAPP* m, int narg, char** arg) : Min_CG(m, narg, arg) {}
    int code() const { return err; }
    double energy() const { return curr_energy; }
};

/* the reference BDF clock with its protected time exposed */
struct BdfRun : public Clock_BDF {
    BdfRun(MAPP* m, int narg, char** arg) : Clock_BDF(m, narg, arg) {}
    double time() const { return t[0]; }
};

struct Harness {
    MAPP* mapp = nullptr;
    VecLst* vecs = nullptr;
    int f_n = -1;
    int dmd = 0;
    int x_dim = 3;
    int nt = 1;
};

Harness H;

void write_raw(const std::string& path, const void* p, size_t bytes)
{
    FILE* fp = fopen(path.c_str(), "wb");
    if (!fp) { fprintf(stderr, "harness: cannot write %s\n", path.c_str()); exit(2); }
    if (bytes) fwrite(p, 1, bytes, fp);
    fclose(fp);
}

std::vector<char> read_raw(const std::string& path)
{
    std::ifstream in(path, std::ios::binary);
    if (!in) { fprintf(stderr, "harness: cannot read %s\n", path.c_str()); exit(2); }
    return std::vector<char>((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
}

void meta(const std::string& prefix, const char* fmt, ...)
{
    FILE* fp = fopen((prefix + ".meta").c_str(), "a");
    va_list ap;
    va_start(ap, fmt);
    vfprintf(fp, fmt, ap);
    va_end(ap);
    fputc('\n', fp);
    fclose(fp);
}

template <class T>
T* vec(const char* name)
{
    T* p = nullptr;
    H.mapp->atoms->vectors[H.mapp->atoms->find(name)].ret(p);
    return p;
}

std::vector<char*> split_args(const std::string& s)
{
    std::vector<char*> out;
    std::istringstream is(s);
    std::string tok;
    while (is >> tok) out.push_back(strdup(tok.c_str()));
    return out;
}

void do_script(const std::string& path)
{
    char prog[] = "mapp", flag[] = "-i";
    std::vector<char> p(path.begin(), path.end());
    p.push_back('\0');
    char* argv[] = {prog, flag, p.data()};
    H.mapp = new MAPP(3, argv, MPI_COMM_WORLD);
    H.dmd = (H.mapp->mode == DMD);
    H.x_dim = H.mapp->atoms->vectors[0].dim;
    H.nt = H.mapp->atom_types->no_types;
}

void do_oracle_ff(const std::string& style)
{
    ForceField* ff = nullptr;
    if (style == "DMD_I") ff = new OracleDMD<ForceField_DMD_I>(H.mapp, true);
    else if (style == "DMD") ff = new OracleDMD<ForceField_DMD>(H.mapp, true);
    else if (style == "DMD_II") ff = new OracleDMD<ForceField_DMD_II>(H.mapp, false);
    else { fprintf(stderr, "harness: unknown oracle style %s\n", style.c_str()); exit(2); }
    if (H.mapp->forcefield) delete H.mapp->forcefield;
    H.mapp->forcefield = ff;
}

/* logging hooks of whichever OracleDMD<Base> is installed */
template <class Base>
bool set_log(ForceField* ff, std::vector<double>* log, long* n_energy_out)
{
    OracleDMD<Base>* o = dynamic_cast<OracleDMD<Base>*>(ff);
    if (!o) return false;
    if (n_energy_out) *n_energy_out = o->n_energy;
    o->force_log = log;
    if (log) o->n_energy = 0;
    return true;
}

bool ff_log(std::vector<double>* log, long* n_energy_out)
{
    ForceField* ff = H.mapp->forcefield;
    return set_log<ForceField_DMD_I>(ff, log, n_energy_out) || set_log<ForceField_DMD>(ff, log, n_energy_out) ||
           set_log<ForceField_DMD_II>(ff, log, n_energy_out);
}

/* Min_LBFGS (min_l-bfgs.cpp) run on the scripted system: init, run, fin.
   Writes the final owned x, the energy of every force_calc (init first, then
   one per iteration) and the result code. */
void do_lbfgs(int m, int max_iter, double etol, const std::string& prefix)
{
    char buf[64];
    snprintf(buf, sizeof(buf), "%.17g", etol);
    std::vector<std::string> a = {"min", "l-bfgs", "m", std::to_string(m), "max_iteration", std::to_string(max_iter),
                                  "energy_tol", buf};
    std::vector<char*> argv;
    for (auto& t : a) argv.push_back(strdup(t.c_str()));
    std::vector<double> log;
    if (!ff_log(&log, nullptr)) { fprintf(stderr, "harness: lbfgs needs an oracle DMD force field\n"); exit(2); }
    LbfgsRun* mn = new LbfgsRun(H.mapp, (int)argv.size(), argv.data());
    mn->init();
    mn->run();
    long n_energy = 0;
    ff_log(nullptr, &n_energy);
    Atoms* atoms = H.mapp->atoms;
    double* x = vec<double>("x");
    write_raw(prefix + ".x.bin", x, sizeof(double) * (size_t)atoms->natms * H.x_dim);
    write_raw(prefix + ".ehist.bin", log.data(), sizeof(double) * log.size());
    meta(prefix, "code %d", mn->code());
    meta(prefix, "energy %.17g", mn->energy());
    meta(prefix, "n_force %d", (int)log.size());
    meta(prefix, "n_energy %ld", n_energy);
    mn->fin();
    delete mn;
    for (char* t : argv) free(t);
}

/* Min_CG (min_cg.cpp) run on the scripted system, outputs as do_lbfgs */
void do_cg(int max_iter, double etol, const std::string& prefix)
{
    char buf[64];
    snprintf(buf, sizeof(buf), "%.17g", etol);
    std::vector<std::string> a = {"min", "cg", "max_iteration", std::to_string(max_iter), "energy_tol", buf};
    std::vector<char*> argv;
    for (auto& t : a) argv.push_back(strdup(t.c_str()));
    std::vector<double> log;
    if (!ff_log(&log, nullptr)) { fprintf(stderr, "harness: cg needs an oracle DMD force field\n"); exit(2); }
    CgRun* mn = new CgRun(H.mapp, (int)argv.size(), argv.data());
    mn->init();
    mn->run();
    long n_energy = 0;
    ff_log(nullptr, &n_energy);
    Atoms* atoms = H.mapp->atoms;
    double* x = vec<double>("x");
    write_raw(prefix + ".x.bin", x, sizeof(double) * (size_t)atoms->natms * H.x_dim);
    write_raw(prefix + ".ehist.bin", log.data(), sizeof(double) * log.size());
    meta(prefix, "code %d", mn->code());
    meta(prefix, "energy %.17g", mn->energy());
    meta(prefix, "n_force %d", (int)log.size());
    meta(prefix, "n_energy %ld", n_energy);
    mn->fin();
    delete mn;
    for (char* t : argv) free(t);
}

void do_ffcoef(const std::string& rest)
{
    std::vector<char*> a = split_args(rest);
    H.mapp->forcefield->coef((int)a.size(), a.data());
    for (char* s : a) free(s);
}

void do_init()
{
    Atoms* atoms = H.mapp->atoms;
    int c_type_n = H.dmd ? atoms->find("c") : atoms->find("type");
    H.f_n = atoms->find_exist("f");
    if (H.f_n < 0) H.f_n = atoms->add<double>(0, H.x_dim, "f");
    int id_n = atoms->find("id");
    int lst[4] = {0, c_type_n, id_n, H.f_n};
    H.vecs = new VecLst(H.mapp, lst, 4);
    H.vecs->add_update(0);
    atoms->reset_comm(H.vecs);
    H.mapp->forcefield->init();
    atoms->ph_setup(1, H.vecs);
    H.mapp->neighbor->init();
    H.mapp->neighbor->create_list(0, 1);
    atoms->store_0();
}

void dump_state(const std::string& prefix)
{
    Atoms* atoms = H.mapp->atoms;
    Neighbor* nb = H.mapp->neighbor;
    int natms = atoms->natms, nph = atoms->natms_ph;
    double* x = vec<double>("x");
    write_raw(prefix + ".x.bin", x, sizeof(double) * (size_t)(natms + nph) * H.x_dim);
    if (atoms->find_exist("x_d") >= 0) {  // MD velocities as read from the CFG
        double* xd = vec<double>("x_d");
        write_raw(prefix + ".xd.bin", xd, sizeof(double) * (size_t)natms * 3);
    }
    if (!H.dmd) {
        int* type = vec<int>("type");
        write_raw(prefix + ".type.bin", type, sizeof(int) * (size_t)(natms + nph));
    } else {
        double* c = vec<double>("c");
        write_raw(prefix + ".c.bin", c, sizeof(double) * (size_t)(natms + nph) * H.nt);
    }
    std::vector<int> sizes(natms), flat;
    for (int i = 0; i < natms; i++) {
        sizes[i] = nb->neighbor_list_size[i];
        for (int k = 0; k < sizes[i]; k++) flat.push_back(nb->neighbor_list[i][k]);
    }
    write_raw(prefix + ".nsize.bin", sizes.data(), sizeof(int) * sizes.size());
    write_raw(prefix + ".nlist.bin", flat.data(), sizeof(int) * flat.size());
    int* id = vec<int>("id");
    write_raw(prefix + ".id.bin", id, sizeof(int) * (size_t)(natms + nph));
    meta(prefix, "natms %d", natms);
    meta(prefix, "natms_ph %d", nph);
    meta(prefix, "no_pairs %d", nb->no_pairs);
    meta(prefix, "x_dim %d", H.x_dim);
    meta(prefix, "nt %d", H.nt);
    for (int i = 0; i < 3; i++)
        meta(prefix, "H%d %.17g %.17g %.17g", i, atoms->H[i][0], atoms->H[i][1], atoms->H[i][2]);
    for (int i = 0; i < 3; i++)
        meta(prefix, "B%d %.17g %.17g %.17g", i, atoms->B[i][0], atoms->B[i][1], atoms->B[i][2]);
    meta(prefix, "cut_ph_s %.17g %.17g %.17g", atoms->cut_ph_s[0], atoms->cut_ph_s[1], atoms->cut_ph_s[2]);
}

void do_force(int st_clc, const std::string& prefix)
{
    Atoms* atoms = H.mapp->atoms;
    double* f = nullptr;
    atoms->vectors[H.f_n].ret(f);
    for (int i = 0; i < H.x_dim * atoms->natms; i++) f[i] = 0.0;
    double en[7] = {0, 0, 0, 0, 0, 0, 0};
    H.mapp->forcefield->force_calc(st_clc, en);
    atoms->vectors[H.f_n].ret(f);
    write_raw(prefix + ".f.bin", f, sizeof(double) * (size_t)atoms->natms * H.x_dim);
    if (H.dmd) {
        int nall = atoms->natms + atoms->natms_ph;
        write_raw(prefix + ".E.bin", vec<double>("E"), sizeof(double) * (size_t)atoms->natms * H.nt);
        write_raw(prefix + ".dE.bin", vec<double>("dE"), sizeof(double) * (size_t)nall * H.nt);
    }
    meta(prefix, "en %.17g %.17g %.17g %.17g %.17g %.17g %.17g", en[0], en[1], en[2], en[3], en[4], en[5], en[6]);
}

void do_energy(const std::string& prefix)
{
    double e = H.mapp->forcefield->energy_calc();
    meta(prefix, "energy %.17g", e);
}

void do_crd(const std::string& prefix)
{
    Atoms* atoms = H.mapp->atoms;
    H.mapp->forcefield->create_2nd_neigh_lst();
    int nall = atoms->natms + atoms->natms_ph;
    write_raw(prefix + ".crd.bin", vec<int>("crd"), sizeof(int) * (size_t)nall);
}

void do_cdot(const std::string& prefix)
{
    Atoms* atoms = H.mapp->atoms;
    H.mapp->forcefield->c_d_calc();
    int natms = atoms->natms, nall = natms + atoms->natms_ph;
    write_raw(prefix + ".c_d.bin", vec<double>("c_d"), sizeof(double) * (size_t)natms * H.nt);
    write_raw(prefix + ".n.bin", vec<double>("n"), sizeof(double) * (size_t)nall * H.nt);
    write_raw(prefix + ".E.bin", vec<double>("E"), sizeof(double) * (size_t)natms * H.nt);
}

void do_calcg(int chk, double alpha, const std::string& apath, const std::string& prefix)
{
    Atoms* atoms = H.mapp->atoms;
    int natms = atoms->natms;
    std::vector<char> raw = read_raw(apath);
    std::vector<double> a((size_t)natms * H.nt), g((size_t)natms * H.nt, 0.0);
    memcpy(a.data(), raw.data(), a.size() * sizeof(double));
    double cost = H.mapp->forcefield->calc_g(chk, alpha, a.data(), g.data());
    meta(prefix, "cost %.17g", cost);
    if (!chk) write_raw(prefix + ".g.bin", g.data(), g.size() * sizeof(double));
}

void do_setx(const std::string& path, const std::string& prefix)
{
    Atoms* atoms = H.mapp->atoms;
    std::vector<char> raw = read_raw(path);
    double* x = vec<double>("x");
    size_t n = (size_t)atoms->natms * H.x_dim;
    memcpy(x, raw.data(), n * sizeof(double));
    /* update_0 rewrites x_0 (vector 1) only when it rebuilds (atoms.cpp:1842-1853) */
    double* x0 = nullptr;
    atoms->vectors[1].ret(x0);
    int d0 = atoms->vectors[1].dim;
    std::vector<double> before(x0, x0 + (size_t)atoms->natms * d0);
    atoms->update_0(0, 1, H.vecs);
    atoms->vectors[1].ret(x0);
    int rebuilt = 0;
    for (size_t k = 0; k < before.size(); k++)
        if (before[k] != x0[k]) { rebuilt = 1; break; }
    meta(prefix, "rebuilt %d", rebuilt);
}

void do_setc(const std::string& path)
{
    Atoms* atoms = H.mapp->atoms;
    std::vector<char> raw = read_raw(path);
    double* c = vec<double>("c");
    memcpy(c, raw.data(), sizeof(double) * (size_t)atoms->natms * H.nt);
    atoms->update(atoms->find("c"));
}

void do_time(const std::string& what, int reps, const std::string& prefix)
{
    Atoms* atoms = H.mapp->atoms;
    double* f = nullptr;
    double en[7];
    double t0 = MPI_Wtime();
    for (int r = 0; r < reps; r++) {
        if (what == "force") {
            atoms->vectors[H.f_n].ret(f);
            for (int i = 0; i < H.x_dim * atoms->natms; i++) f[i] = 0.0;
            H.mapp->forcefield->force_calc(1, en);
        } else if (what == "energy") {
            H.mapp->forcefield->energy_calc();
        } else if (what == "list") {
            H.mapp->neighbor->create_list(0, 1);
        }
    }
    double t1 = MPI_Wtime();
    meta(prefix, "time_%s %d %.9g", what.c_str(), reps, t1 - t0);
}

/* WriteCFG (write_cfg.cpp) with the default vector set, one file */
void do_writecfg(const std::string& prefix, int step)
{
    std::vector<std::string> a = {"write", "cfg", "1", prefix, "x"};
    if (H.dmd) a.push_back("c");
    std::vector<char*> argv;
    for (auto& t : a) argv.push_back(strdup(t.c_str()));
    WriteCFG* wr = new WriteCFG(H.mapp, (int)argv.size(), argv.data());
    wr->write_file(step);
    delete wr;
    for (char* t : argv) free(t);
}

template <class Base>
bool calc_g_count(ForceField* ff, long* n)
{
    OracleDMD<Base>* o = dynamic_cast<OracleDMD<Base>*>(ff);
    if (!o) return false;
    *n = o->n_calc_g;
    return true;
}

/* Clock_Adams (clock_adams.cpp) run on the scripted DMD system */
void do_adams(int order, int steps, const std::string& dt, const std::string& prefix)
{
    Atoms* atoms = H.mapp->atoms;
    ForceField* ff = H.mapp->forcefield;
    std::vector<std::string> a = {"clock", "adams", std::to_string(order), std::to_string(steps), dt};
    std::vector<char*> argv;
    for (auto& t : a) argv.push_back(strdup(t.c_str()));
    long n0 = 0, n1 = 0;
    calc_g_count<ForceField_DMD_I>(ff, &n0) || calc_g_count<ForceField_DMD>(ff, &n0) ||
        calc_g_count<ForceField_DMD_II>(ff, &n0);
    Clock_Adams* ck = new Clock_Adams(H.mapp, (int)argv.size(), argv.data());
    ck->init();
    double t0 = MPI_Wtime();
    ck->run();
    double t1 = MPI_Wtime();
    calc_g_count<ForceField_DMD_I>(ff, &n1) || calc_g_count<ForceField_DMD>(ff, &n1) ||
        calc_g_count<ForceField_DMD_II>(ff, &n1);
    write_raw(prefix + ".c.bin", vec<double>("c"), sizeof(double) * (size_t)atoms->natms * H.nt);
    meta(prefix, "n_calc_g %ld", n1 - n0);
    meta(prefix, "natms %d", atoms->natms);
    meta(prefix, "time_run %.9g", t1 - t0);
    ck->fin();
    delete ck;
    for (char* t : argv) free(t);
}

/* Clock_BDF (clock_bdf.cpp) "clock bdf steps [key value ...]" run on the
   scripted DMD system */
void do_bdf(int steps, const std::string& opts, const std::string& prefix)
{
    Atoms* atoms = H.mapp->atoms;
    ForceField* ff = H.mapp->forcefield;
    std::vector<std::string> a = {"clock", "bdf", std::to_string(steps)};
    std::istringstream os(opts);
    std::string tok;
    while (os >> tok) a.push_back(tok);
    std::vector<char*> argv;
    for (auto& t : a) argv.push_back(strdup(t.c_str()));
    long n0 = 0, n1 = 0;
    calc_g_count<ForceField_DMD_I>(ff, &n0) || calc_g_count<ForceField_DMD>(ff, &n0) ||
        calc_g_count<ForceField_DMD_II>(ff, &n0);
    BdfRun* ck = new BdfRun(H.mapp, (int)argv.size(), argv.data());
    ck->init();
    double t0 = MPI_Wtime();
    ck->run();
    double t1 = MPI_Wtime();
    calc_g_count<ForceField_DMD_I>(ff, &n1) || calc_g_count<ForceField_DMD>(ff, &n1) ||
        calc_g_count<ForceField_DMD_II>(ff, &n1);
    write_raw(prefix + ".c.bin", vec<double>("c"), sizeof(double) * (size_t)atoms->natms * H.nt);
    meta(prefix, "n_calc_g %ld", n1 - n0);
    meta(prefix, "t %.17g", ck->time());
    meta(prefix, "natms %d", atoms->natms);
    meta(prefix, "time_run %.9g", t1 - t0);
    ck->fin();
    delete ck;
    for (char* t : argv) free(t);
}

/* MD_NH (md_nh.cpp) run on the scripted MD-mode system */
void do_md(double t_tar, const std::string& period, int no_it, int no_ch, double dt, double boltz, int seed,
           int steps, const std::string& xd_path, const std::string& prefix)
{
    Atoms* atoms = H.mapp->atoms;
    int natms = atoms->natms;
    if (xd_path != "-") {
        std::vector<char> raw = read_raw(xd_path);
        if (atoms->find_exist("x_d") < 0) atoms->add<double>(0, 3, "x_d");
        double* xd = vec<double>("x_d");
        memcpy(xd, raw.data(), sizeof(double) * (size_t)natms * 3);
    }
    double* x0 = nullptr;
    atoms->vectors[1].ret(x0);
    for (int i = 0; i < natms * atoms->vectors[1].dim; i++) x0[i] = 0.0;
    char tbuf[64];
    snprintf(tbuf, sizeof(tbuf), "%.17g", t_tar);
    std::vector<std::string> a = {"md", "nh", "nvt", "temp", tbuf, period, "eta_iteration", std::to_string(no_it),
                                  "eta_chains", std::to_string(no_ch)};
    if (seed > 0) {
        a.push_back("create_vel");
        a.push_back(std::to_string(seed));
    }
    std::vector<char*> argv;
    for (auto& t : a) argv.push_back(strdup(t.c_str()));
    MD_NH* md = new MD_NH(H.mapp, (int)argv.size(), argv.data());
    md->dt = dt;
    md->boltz = boltz;
    md->init();
    double t0 = MPI_Wtime();
    md->run(steps);
    double t1 = MPI_Wtime();
    write_raw(prefix + ".x.bin", vec<double>("x"), sizeof(double) * (size_t)atoms->natms * 3);
    write_raw(prefix + ".xd.bin", vec<double>("x_d"), sizeof(double) * (size_t)atoms->natms * 3);
    int f_n = atoms->find("f");
    double* f = nullptr;
    atoms->vectors[f_n].ret(f);
    for (int i = 0; i < 3 * atoms->natms; i++) f[i] = 0.0;
    double en[7] = {0, 0, 0, 0, 0, 0, 0};
    H.mapp->forcefield->force_calc(1, en);
    meta(prefix, "en %.17g %.17g %.17g %.17g %.17g %.17g %.17g", en[0], en[1], en[2], en[3], en[4], en[5], en[6]);
    meta(prefix, "natms %d", atoms->natms);
    meta(prefix, "time_run %.9g", t1 - t0);
    md->fin();
    delete md;
    for (char* t : argv) free(t);
}

void run_command(const std::string& line)
{
    std::istringstream is(line);
    std::string cmd;
    if (!(is >> cmd) || cmd[0] == '#') return;
    std::string rest;
    std::getline(is, rest);
    std::istringstream rs(rest);
    if (cmd == "script") { std::string p; rs >> p; do_script(p); }
    else if (cmd == "oracle_ff") { std::string s; rs >> s; do_oracle_ff(s); }
    else if (cmd == "ffcoef") do_ffcoef(rest);
    else if (cmd == "init") do_init();
    else if (cmd == "dump") { std::string p; rs >> p; dump_state(p); }
    else if (cmd == "force") { int s; std::string p; rs >> s >> p; do_force(s, p); }
    else if (cmd == "energy") { std::string p; rs >> p; do_energy(p); }
    else if (cmd == "crd") { std::string p; rs >> p; do_crd(p); }
    else if (cmd == "cdot") { std::string p; rs >> p; do_cdot(p); }
    else if (cmd == "calcg") { int chk; double a; std::string ap, p; rs >> chk >> a >> ap >> p; do_calcg(chk, a, ap, p); }
    else if (cmd == "setx") { std::string xp, p; rs >> xp >> p; do_setx(xp, p); }
    else if (cmd == "setc") { std::string cp; rs >> cp; do_setc(cp); }
    else if (cmd == "cg") { int k; double tol; std::string p; rs >> k >> tol >> p; do_cg(k, tol, p); }
    else if (cmd == "lbfgs") { int m, k; double tol; std::string p; rs >> m >> k >> tol >> p; do_lbfgs(m, k, tol, p); }
    else if (cmd == "writecfg") {
        std::string p;
        int step;
        rs >> p >> step;
        do_writecfg(p, step);
    }
    else if (cmd == "adams") {
        int order, n;
        std::string dt, p;
        rs >> order >> n >> dt >> p;
        do_adams(order, n, dt, p);
    }
    else if (cmd == "bdf") {
        int n;
        std::string p, opts;
        rs >> n >> p;
        std::getline(rs, opts);
        do_bdf(n, opts, p);
    }
    else if (cmd == "md") {
        double T, dt, kb;
        std::string period, xdp, p;
        int it, ch, seed, n;
        rs >> T >> period >> it >> ch >> dt >> kb >> seed >> n >> xdp >> p;
        do_md(T, period, it, ch, dt, kb, seed, n, xdp, p);
    }
    else if (cmd == "time") { std::string w, p; int n; rs >> w >> n >> p; do_time(w, n, p); }
    else { fprintf(stderr, "harness: unknown command %s\n", cmd.c_str()); exit(2); }
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc != 2) { fprintf(stderr, "usage: %s <command-file>\n", argv[0]); return 2; }
    std::ifstream in(argv[1]);
    if (!in) { fprintf(stderr, "harness: cannot open %s\n", argv[1]); return 2; }
    std::string line;
    while (std::getline(in, line)) run_command(line);
    fflush(stdout);
    /* the reference's destructors are not exercised; the process exits here */
    _Exit(0);
}
