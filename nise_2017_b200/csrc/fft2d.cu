// 2D spectra from the 2D response files: the reference's 2DFFT program
// (2DFFT.c:20-830) with the fft x fft transform on the device.
//
// The host part follows the reference's file semantics step for step, because
// users diff these text files:
//  - the keyword file (2DFFT.c:90-234), including "Window" falling through to
//    the following keyword tests and 2DIRraman1/2/3/I/II mapping to 2DIRraman;
//  - one pass per waiting time listed in Waitingtime.dat, or one pass without
//    it (2DFFT.c:252-273);
//  - reading R{par,per,cro}{I,II}[...].dat with the apodisations and the halved
//    t1 = 0 / t3 = 0 borders (:296-361 kI, :459-513 kII); a missing
//    polarisation is skipped;
//  - Rw{par,per,cro}.{I,II}.dat in the reference's quadrant order with its
//    frequency window (:368-438 kI, :514-624 kII), waxis.dat for Matlab;
//  - the sum of rephasing and non-rephasing spectra, 2D.{par,per,cro}.dat, and
//    the broadband pump-probe PP.{par,per,cro}.dat (:626-826), computed from
//    the text just written, as the reference does.  2DIRraman writes the two
//    contributions to separate files instead.
// The arithmetic keeps the reference's types: float inputs and axes, double
// apodisation factors, double transform.
//
// The device part is the forward 2D DFT, exp(-2 pi i (j k / n)) along both
// axes, as two passes of a batched 1D DFT in FP64 with an exact twiddle table
// (twiddle index (j*k) mod n), for any n.
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "nise_b200.h"

extern "C" void nise_set_global_error(const char *msg);

namespace {

// out[b][k] = sum_j in[b][j] w^(jk) for the n rows (es = 1, bs = n) or the n
// columns (es = n, bs = 1) of an n x n array.
__global__ void k_dft_pass(const double2 *in, double2 *out, int n, int es, int bs) {
    extern __shared__ double2 tw[];
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)m / n, &s, &c);
        tw[m] = make_double2(c, s);
    }
    __syncthreads();
    const size_t b = blockIdx.y;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double sr = 0, si = 0;
        int m = 0;  // (j * k) mod n
        for (int j = 0; j < n; j++) {
            double2 z = in[b * bs + (size_t)j * es], w = tw[m];
            sr = fma(z.x, w.x, fma(-z.y, w.y, sr));
            si = fma(z.x, w.y, fma(z.y, w.x, si));
            m += k;
            if (m >= n) m -= n;
        }
        out[b * bs + (size_t)k * es] = make_double2(sr, si);
    }
}

const float c_v = 2.99792458e-5f;                // speed of light in cm/fs, as a float
const float twoPi = (float)(2 * 3.14159265359);  // types.h:7

// The reference's round() macro (2DFFT.c:11) on a float argument.
long round_ref(float x) { return x > 0 ? (long)(x + 0.5) : (long)(x - 0.5); }

struct Input {
    int fft = 0, form = 0, window = 0, raman = 0;
    float deltat = 0, homo = 0, inhomo = 0;
    int tmax1 = 0, tmax2 = 0, tmax3 = 0;
    float min1 = 0, max1 = 0, min2 = 0, max2 = 0, min3 = 0, max3 = 0;
};

bool key(const char *buf, const char *name, size_t len) { return strncmp(buf, name, len) == 0; }

int parse(const char *path, Input &in) {
    FILE *f = fopen(path, "r");
    if (!f) return NISE_ERR_IO;
    char buf[256], word[256];
    while (fgets(buf, sizeof(buf), f)) {
        size_t L = strcspn(buf, " ");
        const char *v = buf + L;
        while (*v == ' ') v++;
        if (key(buf, "FFT", L)) { in.fft = atoi(v); continue; }
        if (key(buf, "Timestep", L)) { in.deltat = (float)atof(v); continue; }
        if (key(buf, "Homogeneous", L)) { in.homo = (float)atof(v); continue; }
        if (key(buf, "Inhomogeneous", L)) { in.inhomo = (float)atof(v); continue; }
        if (key(buf, "Window", L)) {  // no continue here in the reference
            if (sscanf(buf, "%255s %255s", word, word) == 2 && !strcmp(word, "Hann")) in.window = 1;
        }
        if (key(buf, "Format", L)) {
            if (sscanf(buf, "%255s %255s", word, word) == 2) {
                if (!strcmp(word, "Dislin") || !strcmp(word, "Python")) in.form = 0;
                if (!strcmp(word, "Matlab")) in.form = 1;
                if (!strcmp(word, "Gnuplot")) in.form = 2;
            }
            continue;
        }
        if (key(buf, "RunTimes", L)) { sscanf(buf, "RunTimes %d %d %d", &in.tmax1, &in.tmax2, &in.tmax3); continue; }
        if (key(buf, "MinFrequencies", L)) {
            sscanf(buf, "MinFrequencies %f %f %f", &in.min1, &in.min2, &in.min3);
            continue;
        }
        if (key(buf, "MaxFrequencies", L)) {
            sscanf(buf, "MaxFrequencies %f %f %f", &in.max1, &in.max2, &in.max3);
            continue;
        }
        if (key(buf, "Technique", L)) {
            if (sscanf(buf, "Technique %255s", word) == 1)
                in.raman = !strcmp(word, "2DIRraman") || !strcmp(word, "2DIRraman1") || !strcmp(word, "2DIRraman2") ||
                           !strcmp(word, "2DIRraman3") || !strcmp(word, "2DIRramanI") || !strcmp(word, "2DIRramanII");
            continue;
        }
    }
    fclose(f);
    return NISE_OK;
}

// The fft x fft transform on the device; d0/d1 are two n x n work arrays.
int transform(std::vector<double2> &a, int n, double2 *d0, double2 *d1) {
    const size_t bytes = sizeof(double2) * (size_t)n * n;
    const int threads = 128, bx = (n + threads - 1) / threads;
    const size_t sm = sizeof(double2) * n;
    cudaError_t e = cudaMemcpy(d0, a.data(), bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && sm > 48 * 1024)
        e = cudaFuncSetAttribute(k_dft_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) {
        k_dft_pass<<<dim3(bx, n), threads, sm>>>(d0, d1, n, 1, n);  // along the last index (t3)
        k_dft_pass<<<dim3(bx, n), threads, sm>>>(d1, d0, n, n, 1);  // along the first index (t1)
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(a.data(), d0, bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        nise_set_global_error(cudaGetErrorString(e));
        return NISE_ERR_DEVICE;
    }
    return NISE_OK;
}

// Apodise one response value (2DFFT.c:337-353 kI, :489-505 kII): float
// arguments, double factors, the product rounded back to float.
void apodise(const Input &in, int kind, const float *ti, float &rr, float &ir) {
    if (in.homo > 0.0f) {
        double e = exp((double)(-(ti[1] + ti[3]) / 2 / in.homo));
        rr = rr * e;
        ir = ir * e;
    }
    if (in.inhomo > 0.0f) {
        float d = kind == 0 ? ti[1] - ti[3] : ti[1] + ti[3];
        double e = exp((double)(-d * d / 2 / in.inhomo / in.inhomo));
        rr = rr * e;
        ir = ir * e;
    }
    if (in.window == 1) {
        double c1 = cos((double)(ti[1] * twoPi / (4 * in.tmax1 - 4) / in.deltat));
        double c3 = cos((double)(ti[3] * twoPi / (4 * in.tmax3 - 4) / in.deltat));
        rr = rr * c1 * c1;
        rr = rr * c3 * c3;
        ir = ir * c1 * c1;
        ir = ir * c3 * c3;
    }
}

// Read one time-domain file into the transform input; false if it is missing.
bool read_response(const char *name, const Input &in, int kind, std::vector<double2> &a) {
    FILE *f = fopen(name, "r");
    if (!f) return false;
    const long n = in.fft;
    for (auto &z : a) z = make_double2(0.0, 0.0);
    float ti[4] = {0, 0, 0, 0}, rr = 0, ir = 0;
    for (int i = 0; i < in.tmax1; i++)
        for (int k = 0; k < in.tmax3; k++) {
            // the reference does not check this read: a short file repeats the last values
            if (fscanf(f, "%f %f %f %e %e", &ti[1], &ti[2], &ti[3], &rr, &ir) != 5) {
            }
            long index = kind == 0 ? round_ref(ti[3] / in.deltat + n * ti[1] / in.deltat)
                                   : round_ref(ti[3] / in.deltat + n * (ti[1] / in.deltat));
            apodise(in, kind, ti, rr, ir);
            if (i == 0) rr = rr / 2, ir = ir / 2;
            if (k == 0) rr = rr / 2, ir = ir / 2;
            if (index < n * n && index >= 0) {
                if (kind == 0) a[index] = make_double2(rr, ir);
                else a[index] = make_double2(a[index].x + rr, a[index].y + ir);
            }
        }
    fclose(f);
    return true;
}

struct Range { float mi1, ma1, mi3, ma3; };

// Rw*.dat in the reference's quadrant order.  kind 0 (kI, 2DFFT.c:368-438):
// w1 from the negative frequencies; kind 1 (kII, :514-624) tracks the w ranges
// and applies the 2DIRraman w1 offsets.
void write_spectrum(const char *name, const Input &in, int kind, const std::vector<double2> &o, float shift1,
                    float shift3, Range &rng) {
    FILE *out = fopen(name, "w");
    if (!out) return;
    FILE *axis = (kind == 1 && in.form == 1) ? fopen("waxis.dat", "w") : nullptr;
    const int n = in.fft;
    const float sw = 1 / in.deltat / c_v;
    float w1 = 0, w3 = 0;
    for (int half = 0; half < 2; half++) {  // rows n/2..n-1, then 0..n/2-1
        const int i0 = half == 0 ? n / 2 : 0, i1 = half == 0 ? n : n / 2;
        for (int i = i0; i < i1; i++) {
            for (int jh = 0; jh < 2; jh++) {  // columns n/2..n-1, then 0..n/2-1
                const int j0 = jh == 0 ? n / 2 : 0, j1 = jh == 0 ? n : n / 2;
                for (int j = j0; j < j1; j++) {
                    const size_t index = (size_t)j + (size_t)n * i;
                    if (kind == 0) {
                        if (i >= n / 2) w1 = (-n + i) / in.deltat / c_v / n - shift1;
                        if (i < n / 2) w1 = i / in.deltat / c_v / n - shift1;
                        if (j < n / 2) w3 = j / in.deltat / c_v / n - shift3;
                        if (j >= n / 2) w3 = (-n + j) / in.deltat / c_v / n - shift3;
                        if (w1 > -in.max1 && w3 < in.max3 && w1 < -in.min1 && w3 > in.min3) {
                            if (in.form == 0 || in.form == 2) fprintf(out, "%f %f %e %e\n", w1, w3, o[index].x, o[index].y);
                            if (in.form == 1) fprintf(out, "%e ", o[index].y);
                        }
                    } else {
                        if (i >= n / 2) w1 = i / in.deltat / c_v / n + shift1 - sw;
                        if (i < n / 2) w1 = (n + i) / in.deltat / c_v / n + shift1 - sw;
                        if (j < n / 2) w3 = (n + j) / in.deltat / c_v / n + shift3 - sw;
                        if (j >= n / 2) w3 = j / in.deltat / c_v / n + shift3 - sw;
                        if (w1 < in.max1 && w3 < in.max3 && w1 > in.min1 && w3 > in.min3) {
                            if (w1 < rng.mi1) rng.mi1 = w1;
                            if (w1 > rng.ma1) rng.ma1 = w1;
                            if (w3 < rng.mi3) rng.mi3 = w3;
                            if (w3 > rng.ma3) rng.ma3 = w3;
                            // 2DFFT.c:588 offsets w1 by shift3 in this one quadrant
                            if (in.raman) w1 = w1 + ((half == 1 && jh == 0) ? shift3 : shift1);
                            if (in.form == 0 || in.form == 2) fprintf(out, "%f %f %e %e\n", w1, w3, o[index].x, o[index].y);
                            if (in.form == 1) fprintf(out, "%e ", o[index].y);
                        }
                    }
                }
            }
            bool inside = kind == 0 ? (w1 > -in.max1 && w1 < -in.min1) : (w1 < in.max1 && w1 > in.min1);
            if ((in.form == 1 || in.form == 2) && inside) {
                fprintf(out, "\n");
                if (axis) fprintf(axis, "%f\n", w1);
            }
        }
    }
    if (axis) fclose(axis);
    fclose(out);
}

// p1 x p3 text tables of the Rw files, row i = w1 index (1-based in the reference).
struct Table {
    int p1 = 0, p3 = 0;
    std::vector<float> w1, w3, re, im;
    Table(int a, int b) : p1(a), p3(b), w1((size_t)a * b), w3((size_t)a * b), re((size_t)a * b), im((size_t)a * b) {}
    // Read p1 x p3 rows "%f %f %e %e"; entries the file does not hold keep
    // their previous values, as the reference's reused matrices do.
    void read(FILE *f, bool negate_w1) {
        for (int i = 0; i < p1; i++)
            for (int j = 0; j < p3; j++) {
                size_t e = (size_t)i * p3 + j;
                if (fscanf(f, "%f %f %e %e", &w1[e], &w3[e], &re[e], &im[e]) != 4) {
                }
                if (negate_w1) w1[e] = -w1[e];
            }
    }
};

void write_table(const char *name, const Input &in, const Table &axes, const std::vector<float> &re,
                 const std::vector<float> &im) {
    FILE *o = fopen(name, "w");
    if (!o) return;
    for (int k = 0; k < axes.p1; k++) {
        for (int l = 0; l < axes.p3; l++) {
            size_t e = (size_t)k * axes.p3 + l;
            fprintf(o, "%f %f %e %e\n", axes.w1[e], axes.w3[e], re[e], im[e]);
        }
        if (in.form == 2) fprintf(o, "\n");
    }
    fclose(o);
}

// Broadband pump-probe: the float sum over w1 of each w3 column.
void write_pp(const char *name, const std::vector<float> &v, int p1, int p3, const float *axis) {
    FILE *o = fopen(name, "w");
    if (!o) return;
    fprintf(o, "### Broadband pump probe spectrum\n");
    for (int l = 0; l < p3; l++) {
        float pp = 0;
        for (int k = 0; k < p1; k++) pp += v[(size_t)k * p3 + l];
        fprintf(o, "%f %e\n", axis[l], pp);
    }
    fclose(o);
}

// One waiting time (or the only pass when `wt` is null): 2DFFT.c:274-826.
int one_pass(const Input &in, const char *wt, double2 *d0, double2 *d1) {
    const int n = in.fft;
    const char *pol[3] = {"par", "per", "cro"};
    std::vector<double2> a((size_t)n * n);
    float shift1 = 0.5 * (in.min1 + in.max1), shift3 = -0.5 * (in.min3 + in.max3);
    auto names = [&](int p, int kind, char *tname, char *fname) {
        const char *K = kind == 0 ? "I" : "II";
        if (in.raman) {
            snprintf(tname, 256, "R%s%s.IRraman.dat", pol[p], K);
            snprintf(fname, 256, "Rw%sIRraman.%s.dat", pol[p], K);
        } else {
            if (wt) snprintf(tname, 256, "R%s%s_%sfs.dat", pol[p], K, wt);
            else snprintf(tname, 256, "R%s%s.dat", pol[p], K);
            snprintf(fname, 256, "Rw%s.%s.dat", pol[p], K);
        }
    };
    Range unused = {0, 0, 0, 0};
    for (int p = 0; p < 3; p++) {  // kI
        char tname[256], fname[256];
        names(p, 0, tname, fname);
        if (!read_response(tname, in, 0, a)) continue;
        if (int rc = transform(a, n, d0, d1)) return rc;
        write_spectrum(fname, in, 0, a, shift1, shift3, unused);
    }
    shift3 = -shift3;
    Range rng = {shift1, shift1, shift3, shift3};
    for (int p = 0; p < 3; p++) {  // kII; the w ranges restart for every polarisation read
        char tname[256], fname[256];
        names(p, 1, tname, fname);
        if (!read_response(tname, in, 1, a)) continue;
        if (int rc = transform(a, n, d0, d1)) return rc;
        rng = {shift1, shift1, shift3, shift3};
        write_spectrum(fname, in, 1, a, shift1, shift3, rng);
    }
    if (in.form == 1) return NISE_OK;  // Matlab users add the two parts themselves
    const float dw1 = 1 / in.deltat / c_v / n, dw3 = 1 / in.deltat / c_v / n;
    const int p1 = (int)round_ref((rng.ma1 - rng.mi1) / dw1 + 1), p3 = (int)round_ref((rng.ma3 - rng.mi3) / dw3 + 1);
    Table kI(p1, p3), kII(p1, p3);  // reused across the polarisations like the reference's matrices
    std::vector<float> ax3(p3);
    for (int l = 0; l < p3; l++) ax3[l] = rng.mi3 + (rng.ma3 - rng.mi3) * (l + 1) / (p3);
    for (int p = 0; p < 3; p++) {
        char n1[256], n2[256], n2d[256], npp[256], n2d2[256], npp2[256];
        if (in.raman) {
            snprintf(n1, 256, "Rw%sIRraman.I.dat", pol[p]);
            snprintf(n2, 256, "Rw%sIRraman.II.dat", pol[p]);
            snprintf(n2d, 256, "2DIRraman.I.%s.dat", pol[p]);
            snprintf(npp, 256, "PPIRraman.I.%s.dat", pol[p]);
            snprintf(n2d2, 256, "2DIRraman.II.%s.dat", pol[p]);
            snprintf(npp2, 256, "PPIRraman.II.%s.dat", pol[p]);
        } else if (wt) {
            snprintf(n1, 256, "Rw%s.I.dat", pol[p]);
            snprintf(n2, 256, "Rw%s.II.dat", pol[p]);
            snprintf(n2d, 256, "2D.%s_%sfs.dat", pol[p], wt);
            snprintf(npp, 256, "PP.%s_%sfs.dat", pol[p], wt);
        } else {
            snprintf(n1, 256, "Rw%s.I.dat", pol[p]);
            snprintf(n2, 256, "Rw%s.II.dat", pol[p]);
            snprintf(n2d, 256, "2D.%s.dat", pol[p]);
            snprintf(npp, 256, "PP.%s.dat", pol[p]);
        }
        FILE *f = fopen(n1, "r");
        if (!f) continue;
        kI.read(f, true);
        fclose(f);
        if ((f = fopen(n2, "r"))) {
            kII.read(f, false);
            fclose(f);
        }
        if (in.raman) {  // rephasing and non-rephasing stay separate
            write_table(n2d, in, kI, kI.re, kI.im);
            write_table(n2d2, in, kII, kII.re, kII.im);
            std::vector<float> a1(p3), a2(p3);
            for (int l = 0; l < p3; l++) a1[l] = kI.w3[l], a2[l] = kII.w3[l];
            write_pp(npp, kI.im, p1, p3, a1.data());
            write_pp(npp2, kII.im, p1, p3, a2.data());
            continue;
        }
        std::vector<float> IR((size_t)p1 * p3), IRi((size_t)p1 * p3);
        for (int i = 0; i < p1; i++)
            for (int j = 0; j < p3; j++) {
                size_t e = (size_t)i * p3 + j, m = (size_t)(p1 - 1 - i) * p3 + j;
                IR[e] = kI.im[m] + kII.im[e];
                IRi[e] = kI.re[m] + kII.re[e];
            }
        write_table(n2d, in, kII, IRi, IR);
        write_pp(npp, IR, p1, p3, ax3.data());
    }
    return NISE_OK;
}

}  // namespace

extern "C" int nise_2dfft_files(const char *input_path, int device) {
    if (!input_path) {
        nise_set_global_error("nise_2dfft_files: null input path");
        return NISE_ERR_ARG;
    }
    Input in;
    if (parse(input_path, in) != NISE_OK) {
        nise_set_global_error("nise_2dfft_files: input file not found");
        return NISE_ERR_IO;
    }
    if (in.min1 < 0 || in.min2 < 0 || in.min3 < 0 || in.max1 < 0 || in.max2 < 0 || in.max3 < 0) {
        nise_set_global_error("nise_2dfft_files: all field frequencies must be positive");
        return NISE_ERR_ARG;
    }
    if (in.min1 > in.max1 || in.min2 > in.max2 || in.min3 > in.max3) {
        nise_set_global_error("nise_2dfft_files: the max frequency must be larger than the min frequency");
        return NISE_ERR_ARG;
    }
    if (in.fft <= 0 || in.fft > 8192) {
        nise_set_global_error("nise_2dfft_files: FFT keyword not specified (or above 8192)");
        return NISE_ERR_ARG;
    }
    if (!(in.deltat > 0) || in.tmax1 <= 0 || in.tmax3 <= 0) {
        nise_set_global_error("nise_2dfft_files: Timestep and RunTimes are needed");
        return NISE_ERR_ARG;
    }
    double2 *d0 = nullptr, *d1 = nullptr;
    const size_t bytes = sizeof(double2) * (size_t)in.fft * in.fft;
    if (cudaSetDevice(device) != cudaSuccess || cudaMalloc(&d0, bytes) != cudaSuccess ||
        cudaMalloc(&d1, bytes) != cudaSuccess) {
        if (d0) cudaFree(d0);
        nise_set_global_error("nise_2dfft_files: no device or device allocation failed");
        return NISE_ERR_DEVICE;
    }
    int rc = NISE_OK;
    if (access("Waitingtime.dat", F_OK) != -1) {
        FILE *w = fopen("Waitingtime.dat", "r");
        char wt[16];
        while (w && rc == NISE_OK && fscanf(w, "%15s", wt) == 1) rc = one_pass(in, wt, d0, d1);
        if (w) fclose(w);
    } else {
        rc = one_pass(in, nullptr, d0, d1);
    }
    cudaFree(d0);
    cudaFree(d1);
    return rc;
}
