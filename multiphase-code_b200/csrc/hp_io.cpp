// hp_io.cpp -- readers and writers for the reference's file formats, so the
// engine is a drop-in for the same case directories.
//   flow.in            src/sr_Read_flow.F90:19-268
//   grid_procNNNN.dat  src/sr_geometry.F90:101-128
//   bc_procNNNN.in     src/sr_geometry.F90:131-134
//   proc_bcNNNN.in     src/sr_geometry.F90:136-139
//   restartNNNN.in     src/main.F90:427-441 (read), :812-828 (write)
// All reads are list-directed in the reference: one READ statement consumes
// whole records (lines), values separated by blanks or commas, extra values
// on a record ignored, 'd'/'D' accepted as exponent letters.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hydraphase.h"

namespace {

struct LineReader {
    FILE* f = nullptr;
    std::vector<char> buf;
    explicit LineReader(const char* path) : f(std::fopen(path, "rb")), buf(1 << 16) {}
    ~LineReader() { if (f) std::fclose(f); }
    bool ok() const { return f != nullptr; }
    // Reads one record; returns false at end of file.
    bool next(std::string& line) {
        line.clear();
        if (!f) return false;
        bool any = false;
        while (std::fgets(buf.data(), (int)buf.size(), f)) {
            any = true;
            size_t n = std::strlen(buf.data());
            line.append(buf.data(), n);
            if (n && buf[n - 1] == '\n') break;
        }
        while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
        return any;
    }
};

void split_tokens(const std::string& s, std::vector<std::string>& out) {
    out.clear();
    size_t i = 0, n = s.size();
    while (i < n) {
        while (i < n && (s[i] == ' ' || s[i] == '\t' || s[i] == ',')) i++;
        if (i >= n) break;
        size_t j = i;
        while (j < n && !(s[j] == ' ' || s[j] == '\t' || s[j] == ',')) j++;
        out.emplace_back(s.substr(i, j - i));
        i = j;
    }
}

bool parse_real(const std::string& t, double* v) {
    std::string u = t;
    for (char& c : u)
        if (c == 'd' || c == 'D') c = 'e';
    char* end = nullptr;
    errno = 0;
    double x = std::strtod(u.c_str(), &end);
    if (end == u.c_str() || *end != '\0') return false;
    *v = x;
    return true;
}

bool parse_int(const std::string& t, int32_t* v) {
    char* end = nullptr;
    long x = std::strtol(t.c_str(), &end, 10);
    if (end == t.c_str() || *end != '\0') return false;
    *v = (int32_t)x;
    return true;
}

// fast in-place numeric scanning of one record
inline const char* skip_sep(const char* p) {
    while (*p == ' ' || *p == '\t' || *p == ',') p++;
    return p;
}

bool scan_ints(const char* p, int n, int32_t* out) {
    for (int k = 0; k < n; k++) {
        p = skip_sep(p);
        char* end;
        long v = std::strtol(p, &end, 10);
        if (end == p) return false;
        out[k] = (int32_t)v;
        p = end;
    }
    return true;
}

bool scan_reals(const char* p, int n, double* out) {
    for (int k = 0; k < n; k++) {
        p = skip_sep(p);
        char* end;
        double v = std::strtod(p, &end);
        if (end == p) return false;
        if (*end == 'd' || *end == 'D') {   // Fortran exponent letter
            std::string t(p, (const char*)end);
            t.push_back('e');
            const char* q = end + 1;
            while (*q == '+' || *q == '-' || (*q >= '0' && *q <= '9')) t.push_back(*q++);
            v = std::strtod(t.c_str(), nullptr);
            end = const_cast<char*>(q);
        }
        out[k] = v;
        p = end;
    }
    return true;
}

}  // namespace

extern "C" int hp_read_flow(const char* path, hp_params* out) {
    if (!path || !out) return HP_E_ARG;
    LineReader r(path);
    if (!r.ok()) return HP_E_IO;
    hp_params p{};
    // each group: field pointers and kinds (d = real, i = integer)
    struct Item { char kind; void* ptr; };
    std::vector<std::vector<Item>> groups = {
        {{'d', &p.pmax}, {'d', &p.pmin}},
        {{'d', &p.tgmax}, {'d', &p.tgmin}},
        {{'d', &p.ugmax}, {'d', &p.ugmin}},
        {{'d', &p.vgmax}, {'d', &p.vgmin}},
        {{'d', &p.wgmax}, {'d', &p.wgmin}},
        {{'d', &p.upmax}, {'d', &p.upmin}},
        {{'d', &p.vpmax}, {'d', &p.vpmin}},
        {{'d', &p.wpmax}, {'d', &p.wpmin}},
        {{'d', &p.tpmax}, {'d', &p.tpmin}},
        {{'d', &p.pinf}, {'d', &p.gamap}},
        {{'d', &p.gamag}, {'d', &p.cpp}},
        {{'d', &p.cpg}, {'d', &p.amolg}},
        {{'d', &p.prg}, {'d', &p.epslnmax}},
        {{'d', &p.epslnmin}, {'d', &p.epslninf}, {'d', &p.phipzero}},
        {{'d', &p.cfl}, {'i', &p.niter}, {'i', &p.itersub}},
        {{'i', &p.istart}, {'d', &p.diap}},
        {{'d', &p.surfacetension}, {'i', &p.myflux}},
        {{'i', &p.myorder}, {'d', &p.as}, {'d', &p.ts}},
        // read by the five-phase model only; a flow.in may end before them
        {{'d', &p.rhoq}, {'d', &p.rhor}, {'d', &p.rhos}},
        {{'d', &p.radq}, {'d', &p.radr}, {'d', &p.rads}},
        {{'d', &p.phiginit}, {'d', &p.phipinit}, {'d', &p.phiqinit}, {'d', &p.phirinit}, {'d', &p.phisinit}},
    };
    const size_t nrequired = groups.size() - 3;
    std::string line;
    std::vector<std::string> tok;
    size_t gi = 0;
    for (auto& g : groups) {
        bool done = false;
        const bool optional = gi++ >= nrequired;
        while (!done) {
            if (!r.next(line)) {
                if (optional) goto end_of_file;
                return HP_E_IO;   // flow.in ended early
            }
            if (line.find_first_not_of(" \t") == std::string::npos || line[0] == '#') continue;
            size_t c = line.find('#');
            if (c != std::string::npos) line = line.substr(0, c);
            split_tokens(line, tok);
            if (tok.size() < g.size()) continue;
            bool ok = true;
            for (size_t k = 0; k < g.size() && ok; k++) {
                if (g[k].kind == 'd') ok = parse_real(tok[k], (double*)g[k].ptr);
                else ok = parse_int(tok[k], (int32_t*)g[k].ptr);
            }
            done = ok;
        }
    }
end_of_file:
    p.venkat_k = 0.3;
    p.precision = HP_PREC_FP64_PARITY;
    p.renumber = 1;
    p.use_graph = 1;
    *out = p;
    return HP_OK;
}

extern "C" void hp_free_mesh(hp_mesh* m) {
    if (!m) return;
    std::free((void*)m->x); std::free((void*)m->y); std::free((void*)m->z);
    std::free((void*)m->elem); std::free((void*)m->ghost);
    std::memset(m, 0, sizeof *m);
}

extern "C" int hp_read_mesh(const char* case_dir, int32_t rank, hp_mesh* out) {
    if (!case_dir || !out) return HP_E_ARG;
    std::memset(out, 0, sizeof *out);
    char path[4096];
    std::string line;
    int32_t hdr[2];
    // grid
    std::snprintf(path, sizeof path, "%s/geometry_files/grid_proc%04d.dat", case_dir, rank);
    {
        LineReader r(path);
        if (!r.ok() || !r.next(line) || !scan_ints(line.c_str(), 2, hdr)) return HP_E_IO;
        const int nodes = hdr[0], neles = hdr[1];
        if (nodes <= 0 || neles <= 0) return HP_E_IO;
        double* x = (double*)std::calloc(nodes, sizeof(double));
        double* y = (double*)std::calloc(nodes, sizeof(double));
        double* z = (double*)std::calloc(nodes, sizeof(double));
        int32_t* el = (int32_t*)std::calloc((size_t)neles * 9, sizeof(int32_t));
        out->x = x; out->y = y; out->z = z; out->elem = el;
        out->nodes = nodes; out->neles = neles;
        for (int i = 0; i < nodes; i++) {
            int32_t n;
            double v[3];
            if (!r.next(line)) { hp_free_mesh(out); return HP_E_IO; }
            const char* p = line.c_str();
            if (!scan_ints(p, 1, &n)) { hp_free_mesh(out); return HP_E_IO; }
            p = skip_sep(p);
            while (*p && *p != ' ' && *p != '\t' && *p != ',') p++;
            if (!scan_reals(p, 3, v) || n < 1 || n > nodes) { hp_free_mesh(out); return HP_E_IO; }
            x[n - 1] = v[0]; y[n - 1] = v[1]; z[n - 1] = v[2];
        }
        for (int i = 0; i < neles; i++) {
            int32_t v[10];
            if (!r.next(line) || !scan_ints(line.c_str(), 10, v) || v[0] < 1 || v[0] > neles) {
                hp_free_mesh(out);
                return HP_E_IO;
            }
            std::memcpy(el + 9 * (size_t)(v[0] - 1), v + 1, 9 * sizeof(int32_t));
        }
    }
    // boundary ghosts
    std::snprintf(path, sizeof path, "%s/geometry_files/bc_proc%04d.in", case_dir, rank);
    {
        LineReader r(path);
        int32_t ng;
        if (!r.ok() || !r.next(line) || !scan_ints(line.c_str(), 1, &ng) || ng < 0) {
            hp_free_mesh(out);
            return HP_E_IO;
        }
        int32_t* gh = (int32_t*)std::calloc((size_t)ng * 4 + 1, sizeof(int32_t));
        out->ghost = gh;
        out->nghosts = ng;
        for (int i = 0; i < ng; i++) {
            if (!r.next(line) || !scan_ints(line.c_str(), 4, gh + 4 * (size_t)i)) {
                hp_free_mesh(out);
                return HP_E_IO;
            }
        }
    }
    // partition ghosts
    std::snprintf(path, sizeof path, "%s/geometry_files/proc_bc%04d.in", case_dir, rank);
    {
        LineReader r(path);
        int32_t v[2] = {0, 0};
        if (!r.ok() || !r.next(line) || !scan_ints(line.c_str(), 1, v)) { hp_free_mesh(out); return HP_E_IO; }
        out->pghosts = v[0];
    }
    return HP_OK;
}

namespace {
// Record-aware reader of list-directed values: each READ statement starts on
// a new record and skips the rest of its last record.
struct RecordValues {
    LineReader r;
    std::string line;
    explicit RecordValues(const char* p) : r(p) {}
    bool read(size_t n, double* out) {
        size_t got = 0;
        while (got < n) {
            if (!r.next(line)) return false;
            const char* p = line.c_str();
            while (got < n) {
                p = skip_sep(p);
                if (!*p) break;
                char* end;
                double v = std::strtod(p, &end);
                if (end == p) return false;
                out[got++] = v;
                p = end;
            }
        }
        return true;
    }
};
}  // namespace

extern "C" int hp_read_restart(const char* path, int32_t neles, int32_t nghosts, double* time,
                               double* cu_elem, double* ghost_prims) {
    if (!path || neles <= 0 || nghosts < 0) return HP_E_ARG;
    RecordValues rv(path);
    if (!rv.r.ok()) return HP_E_IO;
    double t;
    if (!rv.read(1, &t)) return HP_E_IO;
    std::vector<double> tmp;
    double* cu = cu_elem;
    if (!cu) { tmp.resize((size_t)neles * 10); cu = tmp.data(); }
    if (!rv.read((size_t)neles * 10, cu)) return HP_E_IO;
    std::vector<double> gtmp;
    double* gp = ghost_prims;
    if (!gp) { gtmp.resize((size_t)nghosts * 6 + 1); gp = gtmp.data(); }
    for (int v = 0; v < 6; v++)
        if (nghosts && !rv.read((size_t)nghosts, gp + (size_t)v * nghosts)) return HP_E_IO;
    if (time) *time = t;
    return HP_OK;
}

namespace {
// One restart value: " %25.16E" (26 characters; NaN right-justified).
void put26(double v, char* out) {
    char b[40];
    if (std::isnan(v)) std::snprintf(b, sizeof b, " %25s", "NaN");
    else std::snprintf(b, sizeof b, " %25.16E", v);
    std::memcpy(out, b, 26);
}

// Values of one record, formatted in parallel blocks of fixed-width fields.
bool put_record(FILE* f, const double* v, size_t n, std::vector<char>& buf) {
    const size_t block = (size_t)1 << 20;
    buf.resize(block * 26);
    for (size_t s = 0; s < n; s += block) {
        const long long m = (long long)std::min(block, n - s);
#pragma omp parallel for schedule(static)
        for (long long k = 0; k < m; k++) put26(v[s + k], buf.data() + 26 * k);
        if (std::fwrite(buf.data(), 26, (size_t)m, f) != (size_t)m) return false;
    }
    return std::fputc('\n', f) != EOF;
}
}  // namespace

extern "C" int hp_write_restart(const char* path, int32_t neles, int32_t nghosts, double time,
                                const double* cu_elem, const double* ghost_prims) {
    if (!path || !cu_elem || !ghost_prims) return HP_E_ARG;
    FILE* f = std::fopen(path, "w");
    if (!f) return HP_E_IO;
    std::vector<char> buf;
    bool ok = put_record(f, &time, 1, buf) && put_record(f, cu_elem, (size_t)neles * 10, buf);
    for (int v = 0; v < 6 && ok; v++) ok = put_record(f, ghost_prims + (size_t)v * nghosts, (size_t)nghosts, buf);
    return (std::fclose(f) == 0 && ok) ? HP_OK : HP_E_IO;
}

// ---------------------------------------------------------------------------
// Tecplot file of src/main.F90:956-1268 (two-phase build).  Values go out as
// Fortran ES16.8: one significant digit before the point, eight after, a
// two-digit exponent with its E, or a three-digit exponent without it, right
// in a 16-character field.  Every value line is 17 bytes, so blocks of lines
// are formatted in parallel into a buffer and written in order.
namespace {
void es16_8(double v, char* out) {
    char b[40];
    if (std::isnan(v)) {
        std::snprintf(b, sizeof b, "NaN");
    } else if (std::isinf(v)) {
        std::snprintf(b, sizeof b, v > 0 ? "Infinity" : "-Infinity");
    } else {
        std::snprintf(b, sizeof b, "%.8E", v);
        char* e = std::strchr(b, 'E');
        if (e && std::strlen(e + 2) == 3) std::memmove(e, e + 1, std::strlen(e + 1) + 1);
    }
    const size_t n = std::strlen(b);
    std::memset(out, ' ', 16);
    std::memcpy(out + 16 - n, b, n);
    out[16] = '\n';
}

bool put_column(FILE* f, const double* v, size_t n, std::vector<char>& buf) {
    const size_t block = (size_t)1 << 20;
    buf.resize(block * 17);
    for (size_t s = 0; s < n; s += block) {
        const long long m = (long long)std::min(block, n - s);
#pragma omp parallel for schedule(static)
        for (long long k = 0; k < m; k++) es16_8(v[s + k], buf.data() + 17 * k);
        if (std::fwrite(buf.data(), 17, (size_t)m, f) != (size_t)m) return false;
    }
    return true;
}
}  // namespace

extern "C" int hp_write_tecplot(const char* path, const hp_mesh* mesh, const double* fields) {
    if (!path || !mesh || !fields || !mesh->x || !mesh->y || !mesh->z || !mesh->elem || mesh->neles <= 0 ||
        mesh->nodes <= 0)
        return HP_E_ARG;
    FILE* f = std::fopen(path, "w");
    if (!f) return HP_E_IO;
    const size_t ne = (size_t)mesh->neles, nn = (size_t)mesh->nodes;
    std::fprintf(f, " VARIABLES = \"X\", \"Y\", \"Z\", \"U\",\"V\", \"W\", \"PG\", \"PP\", \"TG\", \"UP\", \"VP\", "
                    "\"WP\", \"PHIG\", \"TP\", \"ROG\", \"ROP\"\n");
    std::fprintf(f, "ZONE ZONETYPE=FETETRAHEDRON, NODES=%zu, ELEMENTS=%zu, DATAPACKING=BLOCK, "
                    "VARLOCATION=([4-16]=CELLCENTERED)\n", nn, ne);
    std::vector<char> buf;
    bool ok = put_column(f, mesh->x, nn, buf) && put_column(f, mesh->y, nn, buf) && put_column(f, mesh->z, nn, buf);
    for (int k = 0; k < 13 && ok; k++) ok = put_column(f, fields + (size_t)k * ne, ne, buf);
    for (size_t e = 0; e < ne && ok; e++) {
        const int32_t* r = mesh->elem + 9 * e;
        ok = std::fprintf(f, "%12d%12d%12d%12d\n", r[0], r[1], r[2], r[3]) > 0;
    }
    return (std::fclose(f) == 0 && ok) ? HP_OK : HP_E_IO;
}
