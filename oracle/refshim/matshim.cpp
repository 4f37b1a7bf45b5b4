// In-memory implementation of the MAT-file API subset declared in mat.h.
//
// Test infrastructure only: it exists so that the reference solver
// (CODE/C++/VS2010/simLB/simLB/cpuLBM.cpp, loadInput at :46-281 and
// createMAT at :467-767) can be compiled unmodified and run as the parity
// oracle.  Instead of MATLAB's .mat format it reads a small container:
//
//   "LBMV1\0\0\0"  u32 nvars
//   per variable:  u32 namelen, name bytes, u32 ndims, u64 dims[ndims],
//                  f64 data[prod(dims)]       (first dimension fastest)
//
// Files opened for writing ("w") are accepted and discarded: the harness
// reads the solver's public arrays directly.
#include "mat.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

struct shim_mxArray {
    std::vector<mwSize> dims;
    std::vector<double> data;
};

struct shim_MATFile {
    bool writing = false;
    std::vector<std::string> names;
    std::vector<shim_mxArray *> vars;
    size_t next = 0;
};

static bool read_exact(FILE *fp, void *dst, size_t n) { return fread(dst, 1, n, fp) == n; }

MATFile *matOpen(const char *filename, const char *mode)
{
    MATFile *m = new shim_MATFile;
    if (mode && mode[0] == 'w') {
        m->writing = true;
        return m;
    }
    FILE *fp = fopen(filename, "rb");
    if (!fp) { delete m; return nullptr; }
    char magic[8];
    uint32_t nvars = 0;
    if (!read_exact(fp, magic, 8) || memcmp(magic, "LBMV1", 5) != 0 || !read_exact(fp, &nvars, 4)) {
        fclose(fp); delete m; return nullptr;
    }
    for (uint32_t v = 0; v < nvars; ++v) {
        uint32_t nl = 0, nd = 0;
        if (!read_exact(fp, &nl, 4)) break;
        std::string name(nl, '\0');
        if (!read_exact(fp, &name[0], nl) || !read_exact(fp, &nd, 4)) break;
        auto *a = new shim_mxArray;
        size_t count = 1;
        for (uint32_t d = 0; d < nd; ++d) {
            uint64_t dim = 0;
            read_exact(fp, &dim, 8);
            a->dims.push_back((mwSize)dim);
            count *= (size_t)dim;
        }
        a->data.resize(count);
        if (count && !read_exact(fp, a->data.data(), count * 8)) { delete a; break; }
        m->names.push_back(name);
        m->vars.push_back(a);
    }
    fclose(fp);
    return m;
}

int matClose(MATFile *pmat)
{
    if (!pmat) return 1;
    for (size_t i = pmat->next; i < pmat->vars.size(); ++i) delete pmat->vars[i];
    delete pmat;
    return 0;
}

char **matGetDir(MATFile *pmat, int *num)
{
    *num = (int)pmat->names.size();
    char **dir = (char **)calloc(pmat->names.size() + 1, sizeof(char *));
    for (size_t i = 0; i < pmat->names.size(); ++i) dir[i] = (char *)pmat->names[i].c_str();
    return dir;
}

mxArray *matGetNextVariable(MATFile *pmat, const char **name)
{
    if (pmat->next >= pmat->vars.size()) return nullptr;
    size_t i = pmat->next++;
    *name = pmat->names[i].c_str();
    return pmat->vars[i];  // ownership passes to the caller (mxDestroyArray)
}

int matPutVariable(MATFile *pmat, const char *name, const mxArray *pa)
{
    (void)pmat; (void)name; (void)pa;
    return 0;
}

mwSize mxGetNumberOfDimensions(const mxArray *pa) { return (mwSize)pa->dims.size(); }
const mwSize *mxGetDimensions(const mxArray *pa) { return pa->dims.data(); }
double *mxGetPr(const mxArray *pa) { return const_cast<double *>(pa->data.data()); }

mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID classid, mxComplexity flag)
{
    (void)classid; (void)flag;
    auto *a = new shim_mxArray;
    size_t count = 1;
    for (mwSize d = 0; d < ndim; ++d) { a->dims.push_back(dims[d]); count *= dims[d]; }
    a->data.assign(count, 0.0);
    return a;
}

void mxDestroyArray(mxArray *pa) { delete pa; }
void mxFree(void *ptr) { free(ptr); }
