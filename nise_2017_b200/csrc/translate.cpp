// Trajectory format translation: the reference's `translate` program
// (translate.c:25-65 driver, transinput :493-598 keywords, readInp :67-237,
// writeOut :239-394, constructHf :396-492, keyWordModify/modifyHam
// :720-940).  Host code only: a job reads one frame per Length from the
// input format, optionally keeps a subset of sites with shifts and isotope
// labels (Modify), builds the two-exciton block when the output carries one,
// and writes the output format.
//
// Formats: GROBIN (int32 tag + float32 records, the engine's own input),
// SKIBIN (GROBIN singles plus per-frame anharmonicity and overtone-dipole
// files, read by Anharmonicfile / Overtonedipolefile), GROASC, MITASC,
// MITTXT and SPECTRON text.  Byte-for-byte behaviour of the reference is
// kept where it is observable: the tag written is the last tag read, GROASC
// writes tag 0, MITASC rows skip one character after each Hamiltonian row,
// text readers keep the last value parsed when a number is missing, binary
// readers keep the previous frame's values past the end of a file.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "nise_b200.h"

extern "C" void nise_set_global_error(const char *msg);

namespace {

enum Fmt { GROBIN, GROASC, MITASC, SPECTRON, MITTXT, SKIBIN, BAD };

Fmt fmt_of(const std::string &s) {
    static const char *names[] = {"GROBIN", "GROASC", "MITASC", "SPECTRON", "MITTXT", "SKIBIN"};
    for (int i = 0; i < 6; i++)
        if (s == names[i]) return (Fmt)i;
    return BAD;
}

const float kSqrt2 = 1.41421356237f;  // the reference's float constant (types.h:10)

// Packed upper-triangle index (Sindex, NISE_subs.h:54-65).
inline int pidx(int a, int b, int n) {
    if (a > b) std::swap(a, b);
    return b + a * ((n << 1) - a - 1) / 2;
}

struct Job {
    std::string io[2][8];  // [in/out][energy, dipole, alpha, anh, over, dx, dy, dz]
    std::string fmt[2], skip;
    int singles = 0, doubles = -1, length = 1;
    float anharmonicity = 16;
    bool modify = false;
    int sel_n = 0, sel_doubles = 0;
    std::vector<int> select, label;
    std::vector<float> shift;
};
enum { E_, D_, AL_, AN_, OV_, DX_, DY_, DZ_ };

// One frame.  The arrays keep their values from frame to frame, as the
// reference's t_ham does.
struct Ham {
    int tag = 0;
    std::vector<float> He, Hf, mu, mu2, anh, over, alpha;
};

struct Files {
    FILE *in[8] = {}, *out[8] = {};
    ~Files() {
        for (int k = 0; k < 8; k++) {
            if (in[k]) fclose(in[k]);
            if (out[k]) fclose(out[k]);
        }
    }
};

int fail(const std::string &msg, int code = NISE_ERR_ARG) {
    nise_set_global_error(msg.c_str());
    return code;
}

// ---------------------------------------------------------------- keywords
// keyWordS/I/F matching (readinput.c:290-360): the line's first token
// (through the first blank) compared by strncmp over its length, first
// keyword in order wins; string values are the second whitespace token.
int parse(const char *path, Job &J) {
    FILE *f = fopen(path, "r");
    if (!f) return fail("File not found!", NISE_ERR_IO);
    static const struct { const char *key; int dir, slot; } files[] = {
        {"InputEnergy", 0, E_}, {"OutputEnergy", 1, E_}, {"InputDipole", 0, D_}, {"OutputDipole", 1, D_},
        {"InputAlpha", 0, AL_}, {"OutputAlpha", 1, AL_}, {"InputAnharm", 0, AN_}, {"OutputAnharm", 1, AN_},
        {"InputOverto", 0, OV_}, {"OutputOverto", 1, OV_}, {"InputDipoleX", 0, DX_}, {"OutputDipoleX", 1, DX_},
        {"InputDipoleY", 0, DY_}, {"OutputDipoleY", 1, DY_}, {"InputDipoleZ", 0, DZ_}, {"OutputDipoleZ", 1, DZ_}};
    char buf[256];
    auto svalue = [&](std::string &dst) {
        char a[256], b[256];
        if (sscanf(buf, "%255s %255s", a, b) == 2) dst = b;
    };
    while (fgets(buf, sizeof(buf), f)) {
        size_t L = strcspn(buf, " ");
        auto is = [&](const char *key) { return strncmp(buf, key, L) == 0; };
        const char *val = buf + L;
        while (*val == ' ') val++;
        bool done = false;
        for (auto &e : files)
            if (is(e.key)) {
                svalue(J.io[e.dir][e.slot]);
                done = true;
                break;
            }
        if (done) continue;
        if (is("Singles")) { J.singles = atoi(val); continue; }
        if (is("Length")) { J.length = atoi(val); continue; }
        if (is("Doubles")) { J.doubles = atoi(val); continue; }
        if (is("Anharmonicity")) { J.anharmonicity = (float)atof(val); continue; }
        if (is("InputFormat")) { svalue(J.fmt[0]); continue; }
        if (is("OutputFormat")) { svalue(J.fmt[1]); continue; }
        if (is("Skip")) { svalue(J.skip); continue; }
        if (strncmp(buf, "Modify", 6) == 0) {  // keyWordModify: three blocks on the following lines
            J.modify = true;
            char line[256], word[256];
            if (!fgets(line, sizeof(line), f) || strncmp(line, "Select", 6)) {
                fclose(f);
                return fail("Select keyword not found after Modify!");
            }
            sscanf(line, "%255s %d", word, &J.sel_n);
            if (J.sel_n < 0) J.sel_n = 0;
            J.sel_doubles = J.skip != "Doubles" ? J.sel_n * (J.sel_n + 1) / 2 : 0;
            J.select.assign(J.sel_n, 0);
            J.label.assign(J.sel_n, 0);
            J.shift.assign(J.sel_n, 0.0f);
            for (int i = 0; i < J.sel_n; i++) {
                if (J.sel_n != J.singles) {
                    if (fscanf(f, "%d ", &J.select[i]) != 1) break;
                } else {
                    J.select[i] = i;
                }
            }
            if (!fgets(line, sizeof(line), f) || strncmp(line, "Label", 5)) {
                fclose(f);
                return fail("Label keyword not found in Modify!");
            }
            for (int i = 0; i < J.sel_n; i++)
                if (fscanf(f, "%d ", &J.label[i]) != 1) break;
            if (!fgets(line, sizeof(line), f) || strncmp(line, "Shift", 5)) {
                fclose(f);
                return fail("Shift keyword not found in Modify!");
            }
            for (int i = 0; i < J.sel_n; i++)
                if (fscanf(f, "%f ", &J.shift[i]) != 1) break;
            continue;
        }
    }
    fclose(f);
    if (J.doubles == -1) J.doubles = J.singles * (J.singles + 1) / 2;  // "standard peptide"
    if (fmt_of(J.fmt[0]) == BAD) return fail("Input format " + J.fmt[0] + " unknown.");
    if (fmt_of(J.fmt[1]) == BAD) return fail("Output format " + J.fmt[1] + " unknown.");
    if (J.singles <= 0) return fail("Singles must be positive");
    if (J.modify && J.sel_n > J.singles) return fail("Modify selects more sites than Singles");
    for (int i = 0; J.modify && i < J.sel_n; i++)
        if (J.select[i] < 0 || J.select[i] >= J.singles) return fail("Modify selects a site out of range");
    return NISE_OK;
}

// ---------------------------------------------------------------- readers
// fread semantics: whole items only, the rest of the destination untouched.
void rd(FILE *f, void *dst, size_t size, size_t n) {
    if (f && n) (void)!fread(dst, size, n, f);
}
void rd_tag(FILE *f, int &tag) {
    int t;
    if (f && fread(&t, sizeof(int), 1, f) == 1) tag = t;
}

// fscanf("%f") keeping the last parsed value when a number is missing.
struct Scan {
    float last = 0;
    float next(FILE *f) {
        float v;
        if (f && fscanf(f, "%f", &v) == 1) last = v;
        return last;
    }
};

// MITASC: one tab-separated line per frame (fgets with the reference's
// 4096-byte buffer); every field is parsed by atof (the reference copies at
// most 16 characters of a field into a blank padded buffer first, which only
// matters for longer fields).  A line past the end of the file leaves the
// values as they were.
struct TabLine {
    char line[4096];
    size_t j = 0, len = 0;
    bool ok = false;
    explicit TabLine(FILE *f) {
        ok = f && fgets(line, sizeof(line), f);
        len = ok ? strlen(line) : 0;
    }
    float next() {
        size_t L = j < len ? strcspn(line + j, "\t") : 0;
        std::string field = j < len ? std::string(line + j, L) : std::string();
        j += L + 1;
        return (float)atof(field.c_str());
    }
};

void read_frame(const Job &J, Fmt in, Files &F, Ham &H) {
    const int N = J.singles, Nd = J.doubles;
    Scan s;
    switch (in) {
    case GROBIN:
        rd_tag(F.in[E_], H.tag);
        rd(F.in[E_], H.He.data(), 4, (size_t)N * (N + 1) / 2);
        rd(F.in[E_], H.Hf.data(), 4, (size_t)Nd * (Nd + 1) / 2);
        rd_tag(F.in[D_], H.tag);
        rd(F.in[D_], H.mu.data(), 4, 3 * (size_t)N);
        rd(F.in[D_], H.mu2.data(), 4, 3 * (size_t)N * Nd);
        if (F.in[AL_]) {
            rd_tag(F.in[AL_], H.tag);
            rd(F.in[AL_], H.alpha.data(), 4, 6 * (size_t)N);
        }
        break;
    case SKIBIN:
        rd_tag(F.in[E_], H.tag);
        rd(F.in[E_], H.He.data(), 4, (size_t)N * (N + 1) / 2);
        rd_tag(F.in[D_], H.tag);
        rd(F.in[D_], H.mu.data(), 4, 3 * (size_t)N);
        rd_tag(F.in[AN_], H.tag);
        rd(F.in[AN_], H.anh.data(), 4, (size_t)N);
        rd_tag(F.in[OV_], H.tag);
        rd(F.in[OV_], H.over.data(), 4, 3 * (size_t)N);
        break;
    case MITASC: {
        // N x N row-major, upper triangle kept; one extra character is
        // skipped after each row of N fields (translate.c:133)
        TabLine e(F.in[E_]);
        if (e.ok)
            for (int k = 0; k < N; k++) {
                for (int l = 0; l < N; l++) {
                    float v = e.next();
                    if (k <= l) H.He[pidx(k, l, N)] = v;
                }
                e.j++;
            }
        for (int x = 0; x < 3; x++) {
            TabLine d(F.in[DX_ + x]);
            if (d.ok)
                for (int k = 0; k < N; k++) H.mu[x * N + k] = d.next();
        }
        break;
    }
    case GROASC: {
        int t;
        if (F.in[E_]) (void)!fscanf(F.in[E_], "%d", &t);  // the tag is read and dropped
        for (int k = 0; k < N; k++)
            for (int l = k; l < N; l++) H.He[pidx(k, l, N)] = s.next(F.in[E_]);
        if (F.in[D_]) (void)!fscanf(F.in[D_], "%d", &t);
        for (int x = 0; x < 3; x++)
            for (int k = 0; k < N; k++) H.mu[x * N + k] = s.next(F.in[D_]);
        if (F.in[AL_]) {
            (void)!fscanf(F.in[AL_], "%d", &t);
            for (int x = 0; x < 6; x++)
                for (int k = 0; k < N; k++) H.alpha[x * N + k] = s.next(F.in[AL_]);
        }
        break;
    }
    case MITTXT:
        for (int k = 0; k < N; k++)
            for (int l = 0; l < N; l++) {
                float v = s.next(F.in[E_]);
                if (k <= l) H.He[pidx(k, l, N)] = v;
            }
        for (int k = 0; k < N; k++)
            for (int x = 0; x < 3; x++) H.mu[x * N + k] = s.next(F.in[D_]);
        break;
    case SPECTRON: {
        char dum[256];
        int t;
        if (F.in[E_]) (void)!fscanf(F.in[E_], "%255s %d", dum, &t);
        for (int k = 0; k < N; k++)
            for (int l = 0; l <= k; l++) H.He[pidx(l, k, N)] = s.next(F.in[E_]);
        if (F.in[D_]) (void)!fscanf(F.in[D_], "%255s %d", dum, &t);
        for (int k = 0; k < N; k++)
            for (int x = 0; x < 3; x++) H.mu[x * N + k] = s.next(F.in[D_]);
        break;
    }
    default: break;
    }
}

// ---------------------------------------------------------------- Modify
// Keep the selected sites in the given order; add the shift and the isotope
// label (1: 13C, -41 cm^-1; 2: 18O, -60 cm^-1) to each kept diagonal.
void select_sites(const Job &J, Ham &H) {
    const int N = J.singles, M = J.sel_n;
    std::vector<float> He((size_t)M * (M + 1) / 2), mu(3 * (size_t)M), over(3 * (size_t)M), anh(M),
        alpha(6 * (size_t)M);
    int e = 0;
    for (int i = 0; i < M; i++) {
        for (int j = i; j < M; j++) {
            float h = H.He[pidx(J.select[i], J.select[j], N)];
            if (i == j) {
                h += J.shift[i];
                if (J.label[i] == 1) h -= 41;
                else if (J.label[i] == 2) h -= 60;
            }
            He[e++] = h;
        }
        anh[i] = H.anh[J.select[i]];
        for (int x = 0; x < 3; x++) {
            mu[x * M + i] = H.mu[x * N + J.select[i]];
            over[x * M + i] = H.over[x * N + J.select[i]];
        }
        for (int x = 0; x < 6; x++) alpha[x * M + i] = H.alpha[x * N + J.select[i]];
    }
    std::copy(He.begin(), He.end(), H.He.begin());
    std::copy(anh.begin(), anh.end(), H.anh.begin());
    std::copy(mu.begin(), mu.end(), H.mu.begin());
    std::copy(over.begin(), over.end(), H.over.begin());
    std::copy(alpha.begin(), alpha.end(), H.alpha.begin());
}

// ---------------------------------------------------------------- doubles
// Two-exciton block of N sites with pair states (a <= b) in packed order:
// energies e_a + e_b (2 e_a - anharmonicity for overtones), couplings J_cd
// between pair states sharing one site (sqrt2 J for an overtone), and the
// singles -> pair dipoles (sqrt2 mu_a into |aa>, mu_b / mu_a into |ab>).
void build_doubles(int N, float A, Ham &H) {
    const int Nf = N * (N + 1) / 2;
    std::vector<int> pa(Nf), pb(Nf);
    for (int a = 0, k = 0; a < N; a++)
        for (int b = a; b < N; b++, k++) pa[k] = a, pb[k] = b;
    const std::vector<float> &He = H.He;
    for (int i = 0; i < Nf; i++) {
        const int a = pa[i], b = pb[i];
        for (int j = i; j < Nf; j++) {
            const int c = pa[j], d = pb[j];
            float w = 0;
            if (i == j) {
                w = a == b ? 2 * He[pidx(a, a, N)] - A : He[pidx(a, a, N)] + He[pidx(b, b, N)];
            } else {
                if (a == b && (c == a || d == a)) w = kSqrt2 * He[pidx(c, d, N)];
                if (c == d && (a == c || b == c)) w = kSqrt2 * He[pidx(a, b, N)];
                if (a != b && c != d) {
                    if (a == c) w = He[pidx(b, d, N)];
                    else if (b == d) w = He[pidx(a, c, N)];
                    else if (a == d) w = He[pidx(c, b, N)];
                    else if (c == b) w = He[pidx(a, d, N)];
                }
            }
            H.Hf[pidx(i, j, Nf)] = w;
        }
    }
    for (int x = 0; x < 3; x++)
        for (int s = 0; s < N; s++)
            for (int j = 0; j < Nf; j++) {
                const int a = pa[j], b = pb[j];
                float w = 0;
                if (a == b) {
                    if (s == a) w = kSqrt2 * H.mu[x * N + s];
                } else {
                    if (a == s) w = H.mu[x * N + b];
                    if (b == s) w = H.mu[x * N + a];
                }
                H.mu2[(size_t)Nf * N * x + (size_t)Nf * s + j] = w;
            }
}

// ---------------------------------------------------------------- writers
void wr(FILE *f, const void *src, size_t size, size_t n) {
    if (f && n) fwrite(src, size, n, f);
}

void write_frame(Fmt out, int N, int Nd, bool doubles, Files &F, const Ham &H, int snapshot) {
    switch (out) {
    case GROBIN:
        wr(F.out[E_], &H.tag, 4, 1);
        wr(F.out[E_], H.He.data(), 4, (size_t)N * (N + 1) / 2);
        if (doubles) wr(F.out[E_], H.Hf.data(), 4, (size_t)Nd * (Nd + 1) / 2);
        wr(F.out[D_], &H.tag, 4, 1);
        wr(F.out[D_], H.mu.data(), 4, 3 * (size_t)N);
        if (doubles) wr(F.out[D_], H.mu2.data(), 4, 3 * (size_t)N * Nd);
        if (F.in[AL_]) {
            wr(F.out[AL_], &H.tag, 4, 1);
            wr(F.out[AL_], H.alpha.data(), 4, 6 * (size_t)N);
        }
        break;
    case SKIBIN:
        wr(F.out[E_], &H.tag, 4, 1);
        wr(F.out[E_], H.He.data(), 4, (size_t)N * (N + 1) / 2);
        wr(F.out[D_], &H.tag, 4, 1);
        wr(F.out[D_], H.mu.data(), 4, 3 * (size_t)N);
        wr(F.out[AN_], &H.tag, 4, 1);
        wr(F.out[AN_], H.anh.data(), 4, (size_t)N);
        wr(F.out[OV_], &H.tag, 4, 1);
        wr(F.out[OV_], H.over.data(), 4, 3 * (size_t)N);
        break;
    case MITASC:
        for (int k = 0; k < N; k++)
            for (int l = 0; l < N; l++) fprintf(F.out[E_], "%f\t", H.He[pidx(k, l, N)]);
        fprintf(F.out[E_], "\n");
        for (int x = 0; x < 3; x++) {
            for (int k = 0; k < N; k++) fprintf(F.out[DX_ + x], "%f\t", H.mu[x * N + k]);
            fprintf(F.out[DX_ + x], "\n");
        }
        break;
    case GROASC:
        fprintf(F.out[E_], "%d ", 0);
        for (int k = 0; k < N; k++)
            for (int l = k; l < N; l++) fprintf(F.out[E_], "%f ", H.He[pidx(k, l, N)]);
        fprintf(F.out[E_], "\n");
        fprintf(F.out[D_], "%d ", 0);
        for (int i = 0; i < 3 * N; i++) fprintf(F.out[D_], "%f ", H.mu[i]);
        fprintf(F.out[D_], "\n");
        if (F.in[AL_]) {
            fprintf(F.out[AL_], "%d ", 0);
            for (int i = 0; i < 6 * N; i++) fprintf(F.out[AL_], "%f ", H.alpha[i]);
            fprintf(F.out[AL_], "\n");
        }
        break;
    case MITTXT:
        for (int k = 0; k < N; k++) {
            for (int l = 0; l < N; l++) fprintf(F.out[E_], "%f ", H.He[pidx(k, l, N)]);
            fprintf(F.out[E_], "\n");
        }
        fprintf(F.out[E_], "\n");
        for (int k = 0; k < N; k++) {
            for (int x = 0; x < 3; x++) fprintf(F.out[D_], "%f ", H.mu[x * N + k]);
            fprintf(F.out[D_], "\n");
        }
        fprintf(F.out[D_], "\n");
        break;
    case SPECTRON:
        fprintf(F.out[E_], "SNAPSHOT %d\n", snapshot + 1);
        for (int k = 0; k < N; k++) {
            for (int l = 0; l <= k; l++) fprintf(F.out[E_], "%f ", H.He[pidx(k, l, N)]);
            fprintf(F.out[E_], "\n");
        }
        fprintf(F.out[D_], "SNAPSHOT %d\n", snapshot + 1);
        for (int k = 0; k < N; k++) {
            for (int x = 0; x < 3; x++) fprintf(F.out[D_], "%f ", H.mu[x * N + k]);
            fprintf(F.out[D_], "\n");
        }
        break;
    default: break;
    }
}

// openInOutput (translate.c:600-700): which files each format uses.
int open_files(const Job &J, Fmt in, Fmt out, Files &F) {
    auto op = [](const std::string &p, const char *mode) { return p.empty() ? nullptr : fopen(p.c_str(), mode); };
    const bool bin_in = in == GROBIN || in == SKIBIN, bin_out = out == GROBIN || out == SKIBIN;
    const char *rm = bin_in ? "rb" : "r", *wm = bin_out ? "wb" : "w";
    F.in[E_] = op(J.io[0][E_], rm);
    if (in == MITASC) {
        for (int s = DX_; s <= DZ_; s++) F.in[s] = op(J.io[0][s], rm);
    } else {
        F.in[D_] = op(J.io[0][D_], rm);
    }
    if (in == GROBIN || in == GROASC) F.in[AL_] = op(J.io[0][AL_], rm);
    if (in == SKIBIN) {
        F.in[AN_] = op(J.io[0][AN_], rm);
        F.in[OV_] = op(J.io[0][OV_], rm);
    }
    F.out[E_] = op(J.io[1][E_], wm);
    if (out == MITASC) {
        for (int s = DX_; s <= DZ_; s++) F.out[s] = op(J.io[1][s], wm);
    } else {
        F.out[D_] = op(J.io[1][D_], wm);
    }
    if ((out == GROBIN || out == GROASC) && F.in[AL_]) F.out[AL_] = op(J.io[1][AL_], wm);
    if (out == SKIBIN) {
        F.out[AN_] = op(J.io[1][AN_], wm);
        F.out[OV_] = op(J.io[1][OV_], wm);
    }
    if (!F.in[E_]) return fail("Problem opening energy input file", NISE_ERR_IO);
    if (!F.out[E_]) return fail("Problem opening energy output file", NISE_ERR_IO);
    if (in == MITASC ? !(F.in[DX_] && F.in[DY_] && F.in[DZ_]) : !F.in[D_])
        return fail("Problem opening dipole input file", NISE_ERR_IO);
    if (out == MITASC ? !(F.out[DX_] && F.out[DY_] && F.out[DZ_]) : !F.out[D_])
        return fail("Problem opening dipole output file", NISE_ERR_IO);
    if (in == SKIBIN && !(F.in[AN_] && F.in[OV_]))
        return fail("Problem opening anharmonicity/overtone input file", NISE_ERR_IO);
    if (out == SKIBIN && !(F.out[AN_] && F.out[OV_]))
        return fail("Problem opening anharmonicity/overtone output file", NISE_ERR_IO);
    if (F.in[AL_] && (out == GROBIN || out == GROASC) && !F.out[AL_])
        return fail("Problem opening polarizability output file", NISE_ERR_IO);
    return NISE_OK;
}

}  // namespace

extern "C" int nise_translate(const char *keyword_file) {
    if (!keyword_file) return fail("null argument");
    Job J;
    int rc = parse(keyword_file, J);
    if (rc) return rc;
    const Fmt in = fmt_of(J.fmt[0]), out = fmt_of(J.fmt[1]);
    Files F;
    if ((rc = open_files(J, in, out, F))) return rc;
    const int N = J.singles, Nf = N * (N + 1) / 2;
    const bool doubles = J.skip != "Doubles";
    Ham H;
    H.He.assign((size_t)Nf, 0.0f);
    // the two-exciton block is sized for N(N+1)/2 pair states (initializeHam,
    // translate.c:870-880); GROBIN input may carry a different Doubles count
    const size_t nd = (size_t)std::max(Nf, J.doubles);
    H.Hf.assign(nd * (nd + 1) / 2, 0.0f);
    H.mu.assign(3 * (size_t)N, 0.0f);
    H.mu2.assign((size_t)N * nd * 3, 0.0f);
    H.anh.assign((size_t)N, 0.0f);
    H.over.assign(3 * (size_t)N, 0.0f);
    H.alpha.assign(6 * (size_t)N, 0.0f);
    for (int t = 0; t < J.length; t++) {
        read_frame(J, in, F, H);
        int n = N, nd_out = J.doubles;
        if (J.modify) {
            select_sites(J, H);
            n = J.sel_n;
            nd_out = J.sel_doubles;
        }
        // constructHf: only when the pair block is the full one (or Modify)
        if (doubles && (J.modify || nd_out == n * (n + 1) / 2)) build_doubles(n, J.anharmonicity, H);
        write_frame(out, n, nd_out, doubles, F, H, t);
    }
    return NISE_OK;
}
