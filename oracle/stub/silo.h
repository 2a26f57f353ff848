// Test infrastructure only (oracle build).  Declarations of the Silo output calls in the
// reference's src/fft.cpp (fft3d2silo, a debugging dump the initial conditions do not call);
// oracle/ic_probe.cpp defines them to abort if reached.
#pragma once
typedef struct DBfile DBfile;
typedef struct DBoptlist DBoptlist;
#define DB_CLOBBER 0
#define DB_LOCAL 0
#define DB_PDB 2
#define DB_FLOAT 19
#define DB_COLLINEAR 130
#define DB_NODECENT 110
DBfile* DBCreateReal(const char* name, int mode, int target, const char* info, int type);
int DBPutQuadmesh(DBfile* db, const char* name, const char* const* coordnames, const void* coords, const int* dims, int ndims, int datatype,
		int coordtype, DBoptlist* opts);
int DBPutQuadvar1(DBfile* db, const char* name, const char* meshname, const void* var, const int* dims, int ndims, const void* mixvar, int mixlen,
		int datatype, int centering, DBoptlist* opts);
int DBClose(DBfile* db);
