/* Minimal stand-in for the c-lime header.
 * The reference's I/O headers (propagator_io.h, contractions_io.h) name the
 * LimeReader/LimeWriter types in prototypes only; the oracle replaces the
 * LIME readers and writers it needs with raw-binary ones (io_shim.cpp), so the
 * types stay opaque and no c-lime routine is declared. */
#ifndef ORACLE_SHIM_LIME_H
#define ORACLE_SHIM_LIME_H
#include <stdint.h>
typedef uint64_t n_uint64_t;
typedef struct oracle_lime_reader LimeReader;
typedef struct oracle_lime_writer LimeWriter;
typedef struct oracle_lime_header LimeRecordHeader;
#define LIME_SUCCESS 0
#define LIME_EOF (-1)
#endif
