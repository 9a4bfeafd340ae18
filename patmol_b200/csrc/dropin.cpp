// dropin.cpp -- the reference's integral and Fock-build entry points
// (twoints.h:14, scfaux.h:22-26, dpmints.h:12, oneints.h:10) on the GPU.
//
// They read the basis through the reference's accessors (basis.h:16-50),
// which the host program defines; the declarations below are weak so that
// the library also loads in programs that have no reference basis module
// (the explicit patgpu_* layer needs none), in which case these entry
// points report the missing accessors through fatalError.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/patgpu.h"

// Layouts of the reference's basis records (shell.h:9-13, center.h:5-7).
typedef struct {
    int npr, lsh, cen, off, nst;
    double *al;
    double *co;
} Shell;
typedef struct {
    double q, r[3];
} Center;

extern "C" {
const Shell *shells() __attribute__((weak));
const Center *centers() __attribute__((weak));
int number_of_shells() __attribute__((weak));
int number_of_centers() __attribute__((weak));
int skip_center() __attribute__((weak));
void fatalError(const char *message) __attribute__((weak));
FILE *createERIFile(int rank, int file_no, const char *bname) __attribute__((weak));   // erifs.c:84-90
// the host's own clean_ERIFS (erifs.c:68-81) compiled under this name
void clean_ERIFS_files(ERIFS *e) __attribute__((weak));
}

namespace {

std::mutex g_lock;
std::map<const ERIFS *, patgpu_handle> g_handles;

[[noreturn]] void die(const char *what)
{
    char buf[768];
    snprintf(buf, sizeof buf, "patgpu: %s: %s", what, patgpu_error_message());
    if (fatalError) fatalError(buf);   // util.c:21-26 prints and exits
    fprintf(stderr, "FATAL ERROR: %s\n", buf);
    exit(EXIT_FAILURE);
}

void need_accessors()
{
    if (!shells || !centers || !number_of_shells || !number_of_centers || !skip_center) {
        fprintf(stderr, "FATAL ERROR: patgpu drop-in entry called without the reference's basis module\n");
        exit(EXIT_FAILURE);
    }
}

// Snapshot of the basis the reference holds right now.
struct Snap {
    std::vector<int> l, cen, off, nst, poff;
    std::vector<double> al, co, q, xyz;
    int nsh = 0, ncen = 0, skip = 0;
};

Snap snapshot()
{
    need_accessors();
    Snap s;
    const Shell *sh = shells();
    const Center *c = centers();
    s.nsh = number_of_shells();
    s.ncen = number_of_centers();
    s.skip = skip_center();
    s.poff.push_back(0);
    for (int i = 0; i < s.nsh; ++i) {
        s.l.push_back(sh[i].lsh);
        s.cen.push_back(sh[i].cen);
        s.off.push_back(sh[i].off);
        s.nst.push_back(sh[i].nst);
        for (int k = 0; k < sh[i].npr; ++k) {
            s.al.push_back(sh[i].al[k]);
            s.co.push_back(sh[i].co[k]);
        }
        s.poff.push_back((int)s.al.size());
    }
    for (int i = 0; i < s.ncen; ++i) {
        s.q.push_back(c[i].q);
        s.xyz.insert(s.xyz.end(), c[i].r, c[i].r + 3);
    }
    return s;
}

// One GPU per MPI rank: the reference's MPI program (patmpi) runs one process
// per rank; pick the device from the launcher's node-local rank.
void select_device_once()
{
    static bool done = false;
    if (done) return;
    done = true;
    const char *vars[] = {"PATGPU_DEVICE", "OMPI_COMM_WORLD_LOCAL_RANK", "MPI_LOCALRANKID", "SLURM_LOCALID",
                          "LOCAL_RANK"};
    for (const char *v : vars) {
        const char *e = getenv(v);
        if (e && *e) {
            patgpu_select_device(atoi(e));
            return;
        }
    }
}

patgpu_handle make_handle(const Snap &s, double tau, int start, int rank, int nproc)
{
    select_device_once();
    patgpu_handle h = nullptr;
    if (patgpu_basis_create_quartets(s.nsh, s.l.data(), s.cen.data(), s.off.data(), s.nst.data(), s.poff.data(),
                                     s.al.data(), s.co.data(), s.ncen, s.q.data(), s.xyz.data(), s.skip, tau, start,
                                     rank, nproc, &h))
        die("building the basis on the GPU");
    return h;
}

bool verbose()
{
    const char *e = getenv("PATGPU_VERBOSE");
    return e && !strcmp(e, "1");
}

double schwarz_tau()
{
    const char *e = getenv("PATGPU_SCHWARZ");
    return e ? atof(e) : 1e-14;
}

}  // namespace

extern "C" {

void two_electron_ints(ERIFS *tfiles, int start)
{
    if (!tfiles) die("two_electron_ints: null handle");
    std::lock_guard<std::mutex> g(g_lock);
    auto it = g_handles.find(tfiles);
    if (it != g_handles.end()) {
        patgpu_basis_destroy(it->second);
        g_handles.erase(it);
    }
    Snap s = snapshot();
    int rank = tfiles->rank, nproc = tfiles->nproc > 0 ? tfiles->nproc : 1;
    tfiles->nfiles = 0;   // integral-direct: no ERI files
    // Every quartet of the set has a shell with index >= start.  When all
    // those shells are component-less (the DPM shells that rhf_dpm_calculation
    // passes at every positron position, rhfscf.c:237), the set is empty: bind
    // no device state and leave G untouched, as the reference's empty XINTS
    // files do.
    bool any = false;
    for (int i = start; i < s.nsh; ++i) any = any || s.nst[i] > 0;
    if (!any) {
        g_handles[tfiles] = nullptr;
        return;
    }
    patgpu_handle h = make_handle(s, schwarz_tau(), start, rank % nproc, nproc);
    g_handles[tfiles] = h;
    // PATGPU_ERI_FILES=1: also write the reference's ERI files, for a host
    // program whose own file-reading G build stays linked
    const char *ef = getenv("PATGPU_ERI_FILES");
    if (ef && !strcmp(ef, "1")) {
        if (!createERIFile) die("PATGPU_ERI_FILES=1 needs the host program's createERIFile");
        int nf = 0;
        if (patgpu_write_eri_files_with(h, start, rank % nproc, nproc, createERIFile, tfiles->basename,
                                        (1LL << 30) / 16, 1 << 20, tfiles->numints, &nf))
            die("two_electron_ints: writing the ERI files");
        tfiles->nfiles = nf;
        long long nrec = 0;
        for (int f = 0; f < nf; ++f) nrec += tfiles->numints[f];
        fprintf(stderr, "patgpu: wrote %d ERI file(s), %lld records\n", nf, nrec);
    }
}

void rhf_form_gmatrix(const ERIFS *tfiles, const double *Pmat, double *Gmat)
{
    std::lock_guard<std::mutex> g(g_lock);
    auto it = g_handles.find(tfiles);
    if (it == g_handles.end()) die("rhf_form_gmatrix before two_electron_ints");
    if (it->second && patgpu_rhf_gmatrix(it->second, Pmat, Gmat)) die("rhf_form_gmatrix");
}

void uhf_form_gmatrix(const ERIFS *tfiles, const double *PmatA, const double *PmatB, double *GmatA, double *GmatB)
{
    std::lock_guard<std::mutex> g(g_lock);
    auto it = g_handles.find(tfiles);
    if (it == g_handles.end()) die("uhf_form_gmatrix before two_electron_ints");
    if (it->second && patgpu_uhf_gmatrix(it->second, PmatA, PmatB, GmatA, GmatB)) die("uhf_form_gmatrix");
}

void momints(void)
{
    select_device_once();
    Snap s = snapshot();
    int n = 0;
    for (int i = 0; i < s.nsh; ++i)
        if (s.nst[i]) n = std::max(n, s.off[i] + s.nst[i]);
    const size_t no2 = (size_t)n * (n + 1) / 2;
    std::vector<double> dip(3 * no2), quad(6 * no2);
    if (patgpu_moments(s.nsh, s.l.data(), s.cen.data(), s.off.data(), s.nst.data(), s.poff.data(), s.al.data(),
                       s.co.data(), s.ncen, s.xyz.data(), dip.data(), quad.data()))
        die("momints");
    // the reference's record stream (momints.c:131-179)
    FILE *f = fopen("MOMINTS.DAT", "wb");
    if (!f) die("momints: cannot create MOMINTS.DAT");
    for (int ish = 0; ish < s.nsh; ++ish)
        for (int jsh = 0; jsh <= ish; ++jsh)
            for (int a = 0; a < s.nst[ish]; ++a) {
                const int ir = s.off[ish] + a;
                for (int b = 0; b < s.nst[jsh]; ++b) {
                    const int jr = s.off[jsh] + b;
                    if (jr > ir) break;
                    const size_t ij = (size_t)ir * (ir + 1) / 2 + jr;
                    double v[9];
                    for (int k = 0; k < 3; ++k) v[k] = dip[k * no2 + ij];
                    for (int k = 0; k < 6; ++k) v[3 + k] = quad[k * no2 + ij];
                    if (fwrite(&ir, sizeof(int), 1, f) != 1 || fwrite(&jr, sizeof(int), 1, f) != 1 ||
                        fwrite(v, sizeof(double), 9, f) != 9)
                        die("momints: writing MOMINTS.DAT");
                }
            }
    if (fclose(f)) die("momints: closing MOMINTS.DAT");
}

void dpm_ints(double *hmat)
{
    select_device_once();
    Snap s = snapshot();
    if (patgpu_onebody(s.nsh, s.l.data(), s.cen.data(), s.off.data(), s.nst.data(), s.poff.data(), s.al.data(),
                       s.co.data(), s.ncen, s.q.data(), s.xyz.data(), s.skip, nullptr, nullptr, nullptr, hmat))
        die("dpm_ints");
}

void one_electron_ints(double *Smat, double *Tmat, double *Hmat)
{
    select_device_once();
    Snap s = snapshot();
    if (patgpu_onebody(s.nsh, s.l.data(), s.cen.data(), s.off.data(), s.nst.data(), s.poff.data(), s.al.data(),
                       s.co.data(), s.ncen, s.q.data(), s.xyz.data(), s.skip, Smat, Tmat, Hmat, nullptr))
        die("one_electron_ints");
}

void clean_ERIFS(ERIFS *e)
{
    if (!e) return;
    size_t left = 0;
    {
        std::lock_guard<std::mutex> g(g_lock);
        auto it = g_handles.find(e);
        if (it != g_handles.end()) {
            if (it->second) patgpu_basis_destroy(it->second);
            g_handles.erase(it);
        }
        left = g_handles.size();
    }
    if (verbose()) fprintf(stderr, "patgpu: clean_ERIFS released the handle's device state, %zu bound\n", left);
    if (clean_ERIFS_files) clean_ERIFS_files(e);
}

void patgpu_release_all(void)
{
    std::lock_guard<std::mutex> g(g_lock);
    for (auto &kv : g_handles)
        if (kv.second) patgpu_basis_destroy(kv.second);
    g_handles.clear();
}

}  // extern "C"
