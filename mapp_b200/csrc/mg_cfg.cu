// Extended / standard CFG configuration files, read as ReadCFG does
// (read_cfg.cpp:225-700): header keys, the box H0 x Transform x basic length
// turned into the lower-triangular H the reference works with, fractional
// positions wrapped into [0, 1), species from the mass / name lines, MD
// velocities (times R, in the frame of the file's box, as the reference
// converts them) and DMD rows (s, alpha per species, c per species).
// The writer restates WriteCFG::write_file (write_cfg.cpp:119-433) for the
// default vector set (x, and c in DMD mode), without auxiliary vectors or id
// sorting.  Host code only, except that mg_cfg_write first reads the
// system's owned state back from the device.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mapp_b200.h"
#include "mg_internal.h"

namespace {

int cfail(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return mg::internal_fail(code, buf);
}

// MAPP::hash_remover (MAPP.cpp:534-558): the line up to '#', tokens joined by
// one space; returns the token count
int hash_remover(const char* line, std::string& out)
{
    out.clear();
    int narg = 0;
    size_t n = strlen(line), cur = 0;
    while (cur < n && line[cur] != '#') {
        if (isspace((unsigned char)line[cur])) {
            cur++;
        } else {
            if (narg) out += ' ';
            while (cur < n && !isspace((unsigned char)line[cur])) out += line[cur++];
            narg++;
        }
    }
    return narg;
}

std::vector<std::string> split(const char* line)
{
    std::string joined;
    hash_remover(line, joined);
    std::vector<std::string> t;
    size_t a = 0;
    while (a < joined.size()) {
        size_t b = joined.find(' ', a);
        if (b == std::string::npos) b = joined.size();
        t.push_back(joined.substr(a, b - a));
        a = b + 1;
    }
    return t;
}

}  // namespace

struct mg_cfg {
    int dmd = 0, nt = 0, natms = 0, vel = 0;
    double H[3][3] = {{0}};
    std::vector<std::string> names;
    std::vector<double> masses;
    std::vector<double> x;   // natms * (3 or 3 + nt)
    std::vector<int> type;   // MD
    std::vector<double> c;   // DMD, natms * nt
    std::vector<double> v;   // MD, natms * 3
};

extern "C" {

int mg_cfg_read(const char* path, int dmd, mg_cfg** out)
{
    if (!path || !out) return cfail(MG_ERR_ARG, "null path or output pointer");
    FILE* fp = fopen(path, "r");
    if (!fp) return cfail(MG_ERR_FILE, "file %s not found", path);
    const int kMax = 4096;
    std::vector<char> line(kMax);
    double H0[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, trns[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    double eta[3][3] = {{0}};
    double basic_length = 1.0, R = 1.0;
    int entry_count = 6, vel_chk = 1, ext_cfg = 0, header_cmplt = 0, declared = -1;
    fpos_t pos;
    auto bad = [&](int code, const char* fmt, const char* arg) {
        fclose(fp);
        return cfail(code, fmt, arg);
    };
    // header (read_cfg.cpp:236-357); the line that ends it is read again as an atom line
    while (!header_cmplt) {
        fgetpos(fp, &pos);
        if (!fgets(line.data(), kMax, fp)) return bad(MG_ERR_FORMAT, "%s: end of file inside the header", path);
        std::string cmd;
        int narg = hash_remover(line.data(), cmd);
        const char* s = cmd.c_str();
        int i, j, n;
        double t;
        char s1[kMax], s2[kMax], s3[kMax];
        if (narg == 0) continue;
        if (narg == 1) {
            if (!strcmp(s, ".NO_VELOCITY.")) {
                vel_chk = 0;
                ext_cfg = 1;
                entry_count -= 3;
            } else if (ext_cfg) {
                header_cmplt = 1;
            } else {
                return bad(MG_ERR_FORMAT, "unknown command: %s", s);
            }
        } else if (narg == 3) {
            if (sscanf(s, "Transform(%d,%d) = %lf", &i, &j, &t) == 3) {
                if (i < 1 || i > 3 || j < 1 || j > 3) return bad(MG_ERR_FORMAT, "unknown component: %s", s);
                trns[i - 1][j - 1] = t;
            } else if (sscanf(s, "eta(%d,%d) = %lf", &i, &j, &t) == 3) {
                if (i < 1 || i > 3 || j < 1 || j > 3) return bad(MG_ERR_FORMAT, "unknown component %s", s);
                eta[i - 1][j - 1] = t;
            } else if (sscanf(s, "entry_count = %d", &n) == 1) {
                entry_count = n;
                ext_cfg = 1;
                if (entry_count < 3 + 3 * vel_chk) return bad(MG_ERR_FORMAT, "wrong number of entry_count%s", "");
            } else {
                return bad(MG_ERR_FORMAT, "unknown command: %s", s);
            }
        } else if (narg == 4) {
            if (sscanf(s, "H0(%d,%d) = %lf A", &i, &j, &t) == 3) {
                if (i < 1 || i > 3 || j < 1 || j > 3) return bad(MG_ERR_FORMAT, "unknown component: %s", s);
                H0[i - 1][j - 1] = t;
            } else if (sscanf(s, "R = %lf %s", &t, s1) == 2) {
                R = t;
            } else if (sscanf(s, "auxiliary[%d] = %s %s", &i, s1, s2) == 3) {
                if (i + 3 + 3 * vel_chk + 1 > entry_count)
                    return bad(MG_ERR_FORMAT, "auxilary component larger than entry_count%s", "");
            } else {
                return bad(MG_ERR_FORMAT, "unknown command: %s", s);
            }
        } else if (narg == 5) {
            if (sscanf(s, "Number of particles = %d", &n) == 1) declared = n;
            else if (sscanf(s, "auxiliary[%d] = %s %s %s", &i, s1, s2, s3) == 4) {
                if (i + 3 + 3 * vel_chk + 1 > entry_count)
                    return bad(MG_ERR_FORMAT, "auxilary component larger than entry_count%s", "");
            } else {
                return bad(MG_ERR_FORMAT, "unknown command: %s", s);
            }
        } else if (narg == 6) {
            if (sscanf(s, "A = %lf Angstrom (basic length-scale)", &t) == 1) basic_length = t;
            else return bad(MG_ERR_FORMAT, "unknown command: %s", s);
        } else if (narg == 8 && ext_cfg == 0) {
            header_cmplt = 1;
        } else {
            return bad(MG_ERR_FORMAT, "unknown command: %s", s);
        }
    }
    fsetpos(fp, &pos);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            if (eta[i][j] != 0.0) return bad(MG_ERR_UNSUPPORTED, "eta(i,j) box strains are not supported%s", "");
    // set_box (read_cfg.cpp:365-458): H_x = H0 Transform, times the basic length;
    // the file's frame is kept for velocities, H becomes lower triangular
    double Hx[3][3] = {{0}};
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) Hx[i][j] += H0[i][k] * trns[k][j];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Hx[i][j] *= basic_length;
    double Hxd[3][3];
    memcpy(Hxd, Hx, sizeof(Hx));
    double det = Hx[0][0] * (Hx[1][1] * Hx[2][2] - Hx[1][2] * Hx[2][1]) -
                 Hx[0][1] * (Hx[1][0] * Hx[2][2] - Hx[1][2] * Hx[2][0]) +
                 Hx[0][2] * (Hx[1][0] * Hx[2][1] - Hx[1][1] * Hx[2][0]);
    if (det == 0) return bad(MG_ERR_FORMAT, "H determinant is zero%s", "");
    double sq[3], Ht[3][3] = {{0}}, b[3];
    for (int i = 0; i < 3; i++) {
        sq[i] = 0.0;
        for (int j = 0; j < 3; j++) sq[i] += Hx[i][j] * Hx[i][j];
    }
    Ht[0][0] = sqrt(sq[0]);
    for (int i = 0; i < 3; i++) Ht[1][0] += Hx[0][i] * Hx[1][i];
    Ht[1][0] /= Ht[0][0];
    Ht[1][1] = sqrt(sq[1] - Ht[1][0] * Ht[1][0]);
    for (int i = 0; i < 3; i++) Ht[2][0] += Hx[0][i] * Hx[2][i];
    Ht[2][0] /= Ht[0][0];
    b[0] = Hx[0][1] * Hx[1][2] - Hx[0][2] * Hx[1][1];
    b[1] = Hx[0][2] * Hx[1][0] - Hx[0][0] * Hx[1][2];
    b[2] = Hx[0][0] * Hx[1][1] - Hx[0][1] * Hx[1][0];
    double babs = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    b[0] /= babs;
    b[1] /= babs;
    b[2] /= babs;
    for (int i = 0; i < 3; i++) Ht[2][2] += Hx[2][i] * b[i];
    Ht[2][1] = sqrt(sq[2] - Ht[2][2] * Ht[2][2] - Ht[2][0] * Ht[2][0]);
    mg_cfg* c = new mg_cfg();
    c->dmd = dmd ? 1 : 0;
    memcpy(c->H, Ht, sizeof(Ht));
    if (c->dmd) {
        if (!ext_cfg) {
            delete c;
            return bad(MG_ERR_FORMAT, "DMD mode can only read extended cfg%s", "");
        }
        if ((entry_count - 3) % 2 != 0) {
            delete c;
            return bad(MG_ERR_FORMAT, "entry_count of a DMD file must be 3 + 2 * species%s", "");
        }
        c->nt = (entry_count - 3) / 2;
    }
    c->vel = (!c->dmd && vel_chk) ? 1 : 0;
    // atom section (read_cfg.cpp:466-580 MD, 584-640 DMD, 644-700 wrap)
    int last_type = -1;
    while (fgets(line.data(), kMax, fp)) {
        std::vector<std::string> a = split(line.data());
        const int narg = (int)a.size();
        if (narg == 0) continue;
        auto add_type = [&](double mass, const std::string& name) {
            for (size_t k = 0; k < c->names.size(); k++)
                if (c->names[k] == name) return (int)k;  // AtomTypes::add_type keeps the first mass
            c->names.push_back(name);
            c->masses.push_back(mass);
            return (int)c->names.size() - 1;
        };
        if (!ext_cfg) {
            if (narg != 8) {
                delete c;
                return bad(MG_ERR_FORMAT, "wrong format: %s", line.data());
            }
            last_type = add_type(atof(a[0].c_str()), a[1]);
            double buf[6];
            for (int i = 0; i < 3; i++) buf[i] = atof(a[i + 2].c_str());
            for (int i = 3; i < 6; i++) buf[i] = atof(a[i + 2].c_str()) * R;
            for (int i = 0; i < 3; i++) {
                while (buf[i] >= 1) buf[i]--;
                while (buf[i] < 0) buf[i]++;
            }
            double vd[3] = {0, 0, 0};
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) vd[j] += buf[i + 3] * Hxd[i][j] * R;
            c->x.insert(c->x.end(), buf, buf + 3);
            c->v.insert(c->v.end(), vd, vd + 3);
            c->type.push_back(last_type);
            continue;
        }
        if (narg == 1) {
            double mass = atof(a[0].c_str());
            if (!fgets(line.data(), kMax, fp)) break;
            std::vector<std::string> nm = split(line.data());
            if (nm.size() != 1) {
                delete c;
                return bad(MG_ERR_FORMAT, "error cfg: %s", line.data());
            }
            if (mass <= 0.0) {
                delete c;
                return bad(MG_ERR_FORMAT, "mass cannot be zero%s", "");
            }
            last_type = add_type(mass, nm[0]);
            if (c->dmd && last_type >= c->nt) {
                delete c;
                return bad(MG_ERR_FORMAT, "exceeded the number of types in DMD%s", "");
            }
            continue;
        }
        if (narg != entry_count) {
            delete c;
            return bad(MG_ERR_FORMAT, "wrong extended format: %s", line.data());
        }
        std::vector<double> buf(entry_count, 0.0);
        if (c->dmd) {
            for (int i = 0; i < entry_count; i++) buf[i] = atof(a[i].c_str());
        } else {
            for (int i = 0; i < 3; i++) buf[i] = atof(a[i].c_str());
            if (vel_chk)
                for (int i = 3; i < 6; i++) buf[i] = atof(a[i].c_str()) * R;
        }
        for (int i = 0; i < 3; i++) {
            while (buf[i] >= 1) buf[i]--;
            while (buf[i] < 0) buf[i]++;
        }
        if (c->dmd) {
            c->x.insert(c->x.end(), buf.begin(), buf.begin() + 3 + c->nt);
            c->c.insert(c->c.end(), buf.begin() + 3 + c->nt, buf.begin() + 3 + 2 * c->nt);
        } else {
            double vd[3] = {0, 0, 0};
            if (vel_chk)
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) vd[j] += buf[i + 3] * Hxd[i][j] * R;
            c->x.insert(c->x.end(), buf.begin(), buf.begin() + 3);
            c->v.insert(c->v.end(), vd, vd + 3);
            c->type.push_back(last_type);
        }
    }
    fclose(fp);
    c->natms = (int)(c->x.size() / (c->dmd ? 3 + c->nt : 3));
    if (declared >= 0 && declared != c->natms) {
        int got = c->natms;
        delete c;
        return cfail(MG_ERR_FORMAT, "%s declares %d particles, lists %d", path, declared, got);
    }
    *out = c;
    return MG_OK;
}

int mg_cfg_info(const mg_cfg* c, int* natms, int* ntypes, double* H, int* has_velocity)
{
    if (!c) return cfail(MG_ERR_ARG, "null mg_cfg");
    if (natms) *natms = c->natms;
    if (ntypes) *ntypes = (int)c->names.size();
    if (H)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) H[3 * i + j] = c->H[i][j];
    if (has_velocity) *has_velocity = c->vel;
    return MG_OK;
}

int mg_cfg_types(const mg_cfg* c, char* names, int name_len, double* masses)
{
    if (!c) return cfail(MG_ERR_ARG, "null mg_cfg");
    for (size_t k = 0; k < c->names.size(); k++) {
        if (names) {
            if ((int)c->names[k].size() >= name_len) return cfail(MG_ERR_ARG, "type name longer than %d", name_len - 1);
            strcpy(names + k * name_len, c->names[k].c_str());
        }
        if (masses) masses[k] = c->masses[k];
    }
    return MG_OK;
}

int mg_cfg_atoms(const mg_cfg* c, double* x_frac, int* type, double* conc, double* velocity)
{
    if (!c) return cfail(MG_ERR_ARG, "null mg_cfg");
    if (x_frac) memcpy(x_frac, c->x.data(), c->x.size() * sizeof(double));
    if (type && !c->dmd) memcpy(type, c->type.data(), c->type.size() * sizeof(int));
    if (conc && c->dmd) memcpy(conc, c->c.data(), c->c.size() * sizeof(double));
    if (velocity && !c->dmd) memcpy(velocity, c->v.data(), c->v.size() * sizeof(double));
    return MG_OK;
}

int mg_cfg_free(mg_cfg* c)
{
    delete c;
    return MG_OK;
}

int mg_cfg_write_arrays(const char* prefix, int step, int dmd, int natms, int ntypes, const char* names,
                        int name_len, const double* masses, const double* H, const double* x, const int* type,
                        const double* conc)
{
    if (!prefix || !names || !masses || !H || (natms > 0 && !x)) return cfail(MG_ERR_ARG, "null argument");
    if (natms < 0 || ntypes < 1 || ntypes > mg::kMaxTypes || name_len < 1) return cfail(MG_ERR_ARG, "bad counts");
    if (natms > 0 && (dmd ? !conc : !type)) return cfail(MG_ERR_ARG, dmd ? "null c" : "null type");
    const int nt = ntypes, x_dim = dmd ? 3 + nt : 3;
    // B = H^-1 as ReadCFG builds it (M3INV, init.h:72-85; read_cfg.cpp:453)
    double A[3][3], B[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) A[i][j] = H[3 * i + j];
    B[0][0] = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    B[1][1] = A[2][2] * A[0][0] - A[2][0] * A[0][2];
    B[2][2] = A[0][0] * A[1][1] - A[0][1] * A[1][0];
    B[1][0] = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    B[2][1] = A[2][0] * A[0][1] - A[2][1] * A[0][0];
    B[0][2] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
    B[2][0] = A[1][0] * A[2][1] - A[2][0] * A[1][1];
    B[0][1] = A[2][1] * A[0][2] - A[0][1] * A[2][2];
    B[1][2] = A[0][2] * A[1][0] - A[1][2] * A[0][0];
    double det = A[0][0] * B[0][0] + A[0][1] * B[1][0] + A[0][2] * B[2][0];
    if (det == 0.0) return cfail(MG_ERR_ARG, "H determinant is zero");
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) B[i][j] /= det;
    std::vector<char> name(name_len + 1, 0);
    auto nm = [&](int t) {
        memcpy(name.data(), names + (size_t)t * name_len, name_len);
        name[name_len] = 0;
        return (const char*)name.data();
    };
    char path[4096];
    snprintf(path, sizeof(path), "%s.%08d.cfg", prefix, step);
    FILE* fp = fopen(path, "w");
    if (!fp) return cfail(MG_ERR_FILE, "cannot open %s", path);
    fprintf(fp, "Number of particles = %d\n", natms);
    fprintf(fp, "A = 1 Angstrom (basic length-scale)\n");
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) fprintf(fp, "H0(%d,%d) = %lf A\n", i + 1, j + 1, H[3 * i + j]);
    fprintf(fp, ".NO_VELOCITY.\n");
    fprintf(fp, "entry_count = %d\n", dmd ? x_dim + nt : 3);
    // x2s_no_correction (atoms.cpp:1901-1920): fractional coordinates, not wrapped
    double row[3 + mg::kMaxTypes];
    auto s_of = [&](int i) {
        const double* xi = x + (size_t)i * x_dim;
        for (int k = 0; k < x_dim; k++) row[k] = xi[k];
        for (int j = 0; j < 3; j++) {
            row[j] = row[j] * B[j][j];
            for (int k = j + 1; k < 3; k++) row[j] += B[k][j] * row[k];
        }
    };
    if (!dmd) {
        for (int t = 0; t < nt; t++) {
            fprintf(fp, "%lf \n%s \n", masses[t], nm(t));
            for (int i = 0; i < natms; i++) {
                if (type[i] != t) continue;
                s_of(i);
                for (int k = 0; k < 3; k++) fprintf(fp, "%lf ", row[k]);
                fprintf(fp, "\n");
            }
        }
        fclose(fp);
        return MG_OK;
    }
    int icomp = 0;
    if (nt == 1) fprintf(fp, "auxiliary[%d] = alpha [reduced unit]\n", icomp++);
    else
        for (int k = 0; k < nt; k++) fprintf(fp, "auxiliary[%d] = alpha_%d [reduced unit]\n", icomp++, k);
    if (nt > 1)
        for (int k = 0; k < nt; k++) fprintf(fp, "auxiliary[%d] = c_%d [reduced unit]\n", icomp++, k);
    else
        fprintf(fp, "auxiliary[%d] = c [reduced unit]\n", icomp++);
    for (int t = 0; t < nt; t++) fprintf(fp, "%lf \n%s \n", masses[t], nm(t));
    for (int i = 0; i < natms; i++) {
        s_of(i);
        for (int k = 0; k < x_dim; k++) fprintf(fp, "%lf ", row[k]);
        for (int k = 0; k < nt; k++) fprintf(fp, "%lf ", conc[(size_t)i * nt + k]);
        fprintf(fp, "\n");
    }
    fclose(fp);
    // the companion .usr file of 1 - c, indexed as the reference indexes it:
    // entry i of the flat natms x nt array for atom i (write_cfg.cpp:415-420)
    snprintf(path, sizeof(path), "%s.%08d.usr", prefix, step);
    FILE* fu = fopen(path, "w");
    if (!fu) return cfail(MG_ERR_FILE, "cannot open %s", path);
    for (int i = 0; i < natms; i++) {
        double tmp = 1.0 - conc[i];
        fprintf(fu, "%f %f %f", tmp, tmp, tmp);
        fprintf(fu, "\n");
    }
    fclose(fu);
    return MG_OK;
}

}  // extern "C"
