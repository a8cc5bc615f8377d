// NISE keyword-file parser with the reference's matching rules
// (readinput.c:13-289): each line's first token (up to the first space) is
// compared with strncmp over the token's own length against the keywords in
// the reference's order, so a prefix of a keyword selects it; the last
// occurrence wins; unknown lines are ignored.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "nise_b200.h"

extern "C" void nise_set_global_error(const char *msg);

namespace {

bool match(const char *buf, const char *key, size_t len) { return strncmp(buf, key, len) == 0; }

const char *value_start(const char *buf, size_t len) {
    const char *p = buf + len;
    while (*p == ' ') p++;
    return p;
}

// keyWordS (readinput.c:292-307): second whitespace token, value kept when absent.
void kw_s(const char *buf, char *value, size_t cap) {
    char dummy[256], v[256];
    if (sscanf(buf, "%255s %255s", dummy, v) == 2) {
        strncpy(value, v, cap - 1);
        value[cap - 1] = 0;
    }
}

}  // namespace

extern "C" int nise_params_default(nise_params *p) {
    if (!p) return NISE_ERR_ARG;
    memset(p, 0, sizeof(*p));
    // readinput.c:24-44
    p->begin = 0;
    p->end = 0;
    p->ts = 5;
    p->anharmonicity = 0;
    p->couplingcut = 0;
    p->fft = 0;
    p->tmax1 = 256;
    p->tmax2 = 0;
    p->tmax3 = 256;
    p->homogen = 0;
    p->inhomogen = 0;
    p->window = 0;
    p->hamiltonian = NISE_HAM_FULL;
    p->propagation = NISE_PROP_SPARSE;
    p->technique = NISE_TECH_OTHER;
    p->temperature = 300;  // readinput.c:32
    p->imag_steps = 0;     // readinput.c:28
    p->precision = NISE_FP32;
    p->launch_mode = NISE_BATCHED;
    p->device = 0;
    return NISE_OK;
}

static int technique_code(const char *t) {
    if (!strcmp(t, "Absorption")) return NISE_TECH_ABSORPTION;
    if (!strcmp(t, "2DIR")) return NISE_TECH_2DIR;
    if (!strcmp(t, "GBIR")) return NISE_TECH_GBIR;
    if (!strcmp(t, "SEIR")) return NISE_TECH_SEIR;
    if (!strcmp(t, "EAIR")) return NISE_TECH_EAIR;
    if (!strcmp(t, "noEAIR")) return NISE_TECH_NOEAIR;
    if (!strcmp(t, "2DUVvis")) return NISE_TECH_2DUVVIS;
    if (!strcmp(t, "GBUVvis")) return NISE_TECH_GBUVVIS;
    if (!strcmp(t, "SEUVvis")) return NISE_TECH_SEUVVIS;
    if (!strcmp(t, "EAUVvis")) return NISE_TECH_EAUVVIS;
    if (!strcmp(t, "noEAUVvis")) return NISE_TECH_NOEAUVVIS;
    if (!strcmp(t, "LD")) return NISE_TECH_LD;
    if (!strcmp(t, "Raman")) return NISE_TECH_RAMAN;
    if (!strcmp(t, "SFG")) return NISE_TECH_SFG;
    if (!strcmp(t, "DOS")) return NISE_TECH_DOS;
    if (!strcmp(t, "CD")) return NISE_TECH_CD;
    // NISE.c:236 (string_in_array)
    if (!strcmp(t, "Luminescence") || !strcmp(t, "PL") || !strcmp(t, "Fluorescence")) return NISE_TECH_LUM;
    return NISE_TECH_OTHER;
}

extern "C" int nise_read_input(const char *path, nise_params *p) {
    if (!path || !p) return NISE_ERR_ARG;
    FILE *f = fopen(path, "r");
    if (!f) {
        nise_set_global_error("input file not found");
        return NISE_ERR_IO;
    }
    char prop[256] = "", window[256] = "", hamiltonian[256] = "Full", technique[256] = "", dummy[256];
    char buf[256];
    while (fgets(buf, sizeof(buf), f)) {
        size_t L = strcspn(buf, " ");
        // Order of readinput.c:76-197.
        if (match(buf, "Propagation", L)) { kw_s(buf, prop, sizeof(prop)); continue; }
        if (match(buf, "Hamiltonianfile", L)) { kw_s(buf, p->energyFName, sizeof(p->energyFName)); continue; }
        if (match(buf, "Dipolefile", L)) { kw_s(buf, p->dipoleFName, sizeof(p->dipoleFName)); continue; }
        if (match(buf, "Alphafile", L)) { kw_s(buf, p->alphaFName, sizeof(p->alphaFName)); continue; }
        if (match(buf, "Anharmonicfile", L)) { kw_s(buf, p->anharFName, sizeof(p->anharFName)); continue; }
        if (match(buf, "Overtonedipolefile", L)) { kw_s(buf, p->overdipFName, sizeof(p->overdipFName)); continue; }
        if (match(buf, "Positionfile", L)) { kw_s(buf, p->positionFName, sizeof(p->positionFName)); continue; }
        if (match(buf, "Couplingfile", L)) { kw_s(buf, p->couplingFName, sizeof(p->couplingFName)); continue; }
        if (match(buf, "PBCfile", L)) { kw_s(buf, p->pbcFName, sizeof(p->pbcFName)); continue; }
        if (match(buf, "SingleShiftfile", L)) {
            kw_s(buf, p->singleShiftFName, sizeof(p->singleShiftFName));
            continue;
        }
        if (match(buf, "Length", L)) { p->length = atoi(value_start(buf, L)); continue; }
        if (match(buf, "Samplerate", L)) { p->sample = atoi(value_start(buf, L)); continue; }
        if (match(buf, "BeginPoint", L)) { p->begin = atoi(value_start(buf, L)); continue; }
        if (match(buf, "EndPoint", L)) { p->end = atoi(value_start(buf, L)); continue; }
        if (match(buf, "Lifetime", L)) { p->lifetime = (float)atof(value_start(buf, L)); continue; }
        if (match(buf, "Homogeneous", L)) { p->homogen = (float)atof(value_start(buf, L)); continue; }
        if (match(buf, "Inhomogeneous", L)) { p->inhomogen = (float)atof(value_start(buf, L)); continue; }
        if (match(buf, "Window", L)) { kw_s(buf, window, sizeof(window)); continue; }
        if (match(buf, "Timestep", L)) { p->deltat = (float)atof(value_start(buf, L)); continue; }
        if (match(buf, "Anharmonicity", L)) { p->anharmonicity = (float)atof(value_start(buf, L)); continue; }
        if (match(buf, "FFT", L)) { p->fft = atoi(value_start(buf, L)); continue; }
        if (match(buf, "Threshold", L)) { p->thres = (float)atof(value_start(buf, L)); continue; }
        if (match(buf, "Couplingcut", L)) { p->couplingcut = (float)atof(value_start(buf, L)); continue; }
        if (match(buf, "Temperature", L)) { p->temperature = (float)atof(value_start(buf, L)); continue; }
        if (match(buf, "RunTimes", L)) {
            sscanf(buf, "%255s %d %d %d", dummy, &p->tmax1, &p->tmax2, &p->tmax3);
            continue;
        }
        if (match(buf, "ImaginaryTimesteps", L)) { p->imag_steps = atoi(value_start(buf, L)); continue; }
        if (match(buf, "Trotter", L)) { p->ts = atoi(value_start(buf, L)); continue; }
        if (match(buf, "Interpolation", L)) continue;
        if (match(buf, "Cluster", L)) continue;
        if (match(buf, "Singles", L)) { p->singles = atoi(value_start(buf, L)); continue; }
        if (match(buf, "Doubles", L)) { p->doubles = atoi(value_start(buf, L)); continue; }
        if (match(buf, "MinFrequencies", L)) {
            sscanf(buf, "%255s %f %f %f", dummy, &p->min1, &p->min2, &p->min3);
            continue;
        }
        if (match(buf, "MaxFrequencies", L)) {
            sscanf(buf, "%255s %f %f %f", dummy, &p->max1, &p->max2, &p->max3);
            continue;
        }
        if (match(buf, "Static", L)) continue;
        if (match(buf, "Technique", L)) { kw_s(buf, technique, sizeof(technique)); continue; }
        if (match(buf, "HamiltonianType", L)) { kw_s(buf, hamiltonian, sizeof(hamiltonian)); continue; }
        if (match(buf, "Basis", L)) continue;
        if (match(buf, "Projection", L)) {
            fclose(f);
            nise_set_global_error("Projection is not supported by this engine");
            return NISE_ERR_UNSUPPORTED;
        }
        if (match(buf, "PrintLevel", L)) continue;
    }
    fclose(f);

    strncpy(p->technique_name, technique, sizeof(p->technique_name) - 1);
    p->technique = technique_code(technique);
    // readinput.c:236-254 (Diagonal accepted here)
    p->propagation = NISE_PROP_SPARSE;
    if (!strcmp(prop, "Coupling")) p->propagation = NISE_PROP_COUPLING;
    if (!strcmp(prop, "Diagonal")) p->propagation = NISE_PROP_DIAGONAL;
    if (!strcmp(prop, "RK4")) p->propagation = NISE_PROP_RK4;
    p->window = !strcmp(window, "Hann") ? 1 : 0;
    if (!strcmp(hamiltonian, "Full")) p->hamiltonian = NISE_HAM_FULL;
    else if (!strcmp(hamiltonian, "Coupling")) p->hamiltonian = NISE_HAM_COUPLING;
    else if (!strcmp(hamiltonian, "TransitionDipole")) p->hamiltonian = NISE_HAM_TDC;
    else if (!strcmp(hamiltonian, "ExtendedDipole")) p->hamiltonian = NISE_HAM_EDC;
    else {
        nise_set_global_error("HamiltonianType not supported by this engine (Full, Coupling, TransitionDipole, "
                              "ExtendedDipole)");
        return NISE_ERR_UNSUPPORTED;
    }
    // readinput.c:206-233
    if (p->technique >= NISE_TECH_2DIR && p->technique <= NISE_TECH_NOEAUVVIS) {
        p->tmax3 = p->tmax1;
        if (p->length < p->tmax1 + p->tmax2 + p->tmax3) {
            nise_set_global_error("The trajectory length is too small");
            return NISE_ERR_ARG;
        }
    } else if (p->length < p->tmax1) {
        nise_set_global_error("The trajectory length is too small");
        return NISE_ERR_ARG;
    }
    if (p->tmax1 == 0) {
        nise_set_global_error("First runtime variable is zero");
        return NISE_ERR_ARG;
    }
    return NISE_OK;
}
