/*
 * Minimal raw-file stand-in for the HDF5 C API, used ONLY to compile the
 * reference SEDI validators (ValidateSolver.hpp, ValidateEstimator.hpp) and
 * Slice3d::dump_hdf5/load_hdf5 (Slice3d.hpp:115-161) unmodified on a machine
 * without libhdf5.  Test infrastructure, not product code.
 *
 * Format ("SEDI raw archive"): the archive path is a directory; each dataset
 * <name> is the file <archive>/<name>.raw holding
 *     char[8] "SEDIRAW1" | u32 ndims | u32 elem_bytes | u64 dims[ndims] | data
 * with data in the row-major order H5Dwrite receives it (Slice3d::pack_into
 * writes i3 fastest, Slice3d.hpp:42-52).  The same format is read and written
 * by the product CLI (-V/-E) and by the Python tests.
 *
 * Only the calls the reference makes are provided: H5Fcreate/Fopen/Fclose,
 * H5Dcreate/Dopen/Dread/Dwrite/Dclose/Dget_space,
 * H5Screate_simple/Sget_simple_extent_ndims/Sget_simple_extent_dims/Sclose.
 */
#ifndef SEDI_ORACLE_SHIM_HDF5_H
#define SEDI_ORACLE_SHIM_HDF5_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdint.h>
#include <string>
#include <sys/stat.h>
#include <sys/types.h>

typedef long long hid_t;
typedef unsigned long long hsize_t;
typedef int herr_t;

#define H5P_DEFAULT ((hid_t)0)
#define H5S_ALL ((hid_t)0)
#define H5F_ACC_RDONLY 0u
#define H5F_ACC_TRUNC 2u
#define H5T_NATIVE_FLOAT ((hid_t)4)
#define H5T_NATIVE_DOUBLE ((hid_t)8)

namespace sedi_h5shim {

struct Space { int used; int ndims; hsize_t dims[8]; };
struct File { int used; std::string path; };
struct Dset { int used; std::string path; int writable; int ndims; hsize_t dims[8]; unsigned elem; };

static Space spaces[64];
static File files[16];
static Dset dsets[64];

static inline void fail(const char *what, const std::string &p) {
	fprintf(stderr, "raw HDF5 stand-in: %s failed for '%s'\n", what, p.c_str());
	exit(2);
}

template <typename T, int N>
static inline int slot(T (&tab)[N]) {
	for (int i = 0; i < N; i++)
		if (!tab[i].used) { tab[i].used = 1; return i; }
	fprintf(stderr, "raw HDF5 stand-in: handle table full\n");
	exit(2);
}

static inline uint64_t count(int nd, const hsize_t *d) {
	uint64_t n = 1;
	for (int i = 0; i < nd; i++) n *= d[i];
	return n;
}

} // namespace sedi_h5shim

static inline hid_t H5Fcreate(const char *name, unsigned, hid_t, hid_t) {
	using namespace sedi_h5shim;
	mkdir(name, 0755);
	struct stat st;
	if (stat(name, &st) != 0 || !S_ISDIR(st.st_mode)) fail("H5Fcreate", name);
	int i = slot(files);
	files[i].path = name;
	return 1000 + i;
}

static inline hid_t H5Fopen(const char *name, unsigned, hid_t) {
	using namespace sedi_h5shim;
	struct stat st;
	if (stat(name, &st) != 0 || !S_ISDIR(st.st_mode)) fail("H5Fopen", name);
	int i = slot(files);
	files[i].path = name;
	return 1000 + i;
}

static inline herr_t H5Fclose(hid_t f) {
	sedi_h5shim::files[f - 1000].used = 0;
	return 0;
}

static inline hid_t H5Screate_simple(int rank, const hsize_t *dims, const hsize_t *) {
	using namespace sedi_h5shim;
	int i = slot(spaces);
	spaces[i].ndims = rank;
	for (int d = 0; d < rank; d++) spaces[i].dims[d] = dims[d];
	return 2000 + i;
}

static inline herr_t H5Sclose(hid_t s) {
	sedi_h5shim::spaces[s - 2000].used = 0;
	return 0;
}

static inline int H5Sget_simple_extent_ndims(hid_t s) { return sedi_h5shim::spaces[s - 2000].ndims; }

static inline int H5Sget_simple_extent_dims(hid_t s, hsize_t *dims, hsize_t *) {
	const sedi_h5shim::Space &sp = sedi_h5shim::spaces[s - 2000];
	for (int d = 0; d < sp.ndims; d++) dims[d] = sp.dims[d];
	return sp.ndims;
}

static inline hid_t H5Dcreate(hid_t f, const char *name, hid_t type, hid_t space, hid_t, hid_t, hid_t) {
	using namespace sedi_h5shim;
	int i = slot(dsets);
	Dset &d = dsets[i];
	d.path = files[f - 1000].path + "/" + name + ".raw";
	d.writable = 1;
	d.elem = (unsigned)type;
	d.ndims = spaces[space - 2000].ndims;
	for (int k = 0; k < d.ndims; k++) d.dims[k] = spaces[space - 2000].dims[k];
	return 3000 + i;
}

static inline hid_t H5Dopen(hid_t f, const char *name, hid_t) {
	using namespace sedi_h5shim;
	int i = slot(dsets);
	Dset &d = dsets[i];
	d.path = files[f - 1000].path + "/" + name + ".raw";
	d.writable = 0;
	FILE *fp = fopen(d.path.c_str(), "rb");
	if (!fp) fail("H5Dopen", d.path);
	char magic[8];
	uint32_t nd = 0, el = 0;
	if (fread(magic, 1, 8, fp) != 8 || memcmp(magic, "SEDIRAW1", 8) != 0) fail("H5Dopen (magic)", d.path);
	if (fread(&nd, 4, 1, fp) != 1 || fread(&el, 4, 1, fp) != 1 || nd > 8) fail("H5Dopen (header)", d.path);
	uint64_t dims[8];
	if (fread(dims, 8, nd, fp) != nd) fail("H5Dopen (dims)", d.path);
	fclose(fp);
	d.ndims = (int)nd;
	d.elem = el;
	for (unsigned k = 0; k < nd; k++) d.dims[k] = dims[k];
	return 3000 + i;
}

static inline hid_t H5Dget_space(hid_t ds) {
	const sedi_h5shim::Dset &d = sedi_h5shim::dsets[ds - 3000];
	return H5Screate_simple(d.ndims, d.dims, 0);
}

static inline herr_t H5Dwrite(hid_t ds, hid_t memtype, hid_t, hid_t, hid_t, const void *buf) {
	using namespace sedi_h5shim;
	Dset &d = dsets[ds - 3000];
	if (!d.writable || (unsigned)memtype != d.elem) fail("H5Dwrite", d.path);
	FILE *fp = fopen(d.path.c_str(), "wb");
	if (!fp) fail("H5Dwrite (open)", d.path);
	uint32_t nd = (uint32_t)d.ndims, el = d.elem;
	uint64_t dims[8];
	for (int k = 0; k < d.ndims; k++) dims[k] = d.dims[k];
	uint64_t n = count(d.ndims, d.dims);
	if (fwrite("SEDIRAW1", 1, 8, fp) != 8 || fwrite(&nd, 4, 1, fp) != 1 || fwrite(&el, 4, 1, fp) != 1 ||
	    fwrite(dims, 8, nd, fp) != nd || fwrite(buf, el, n, fp) != n)
		fail("H5Dwrite (write)", d.path);
	fclose(fp);
	return 0;
}

static inline herr_t H5Dread(hid_t ds, hid_t memtype, hid_t, hid_t, hid_t, void *buf) {
	using namespace sedi_h5shim;
	Dset &d = dsets[ds - 3000];
	if ((unsigned)memtype != d.elem) fail("H5Dread (type)", d.path);
	FILE *fp = fopen(d.path.c_str(), "rb");
	if (!fp) fail("H5Dread (open)", d.path);
	long off = 16 + 8L * d.ndims;
	uint64_t n = count(d.ndims, d.dims);
	if (fseek(fp, off, SEEK_SET) != 0 || fread(buf, d.elem, n, fp) != n) fail("H5Dread (read)", d.path);
	fclose(fp);
	return 0;
}

static inline herr_t H5Dclose(hid_t ds) {
	sedi_h5shim::dsets[ds - 3000].used = 0;
	return 0;
}

#endif
