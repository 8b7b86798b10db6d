/* Prototype-only declarations of the public SQLite C API subset that the
 * reference geo2rdr executable uses (https://sqlite.org/c3ref/intro.html).
 * The system ships libsqlite3.so.0 without its development header; this file
 * lets the reference sources compile against it.  Test infrastructure only:
 * it is used by oracle/build_ref.py to build the reference checker. */
#ifndef S1B_REF_SQLITE3_SHIM_H
#define S1B_REF_SQLITE3_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif
typedef struct sqlite3 sqlite3;
typedef struct sqlite3_stmt sqlite3_stmt;
typedef void (*sqlite3_destructor_type)(void *);
#define SQLITE_OK 0
#define SQLITE_ROW 100
#define SQLITE_STATIC ((sqlite3_destructor_type)0)
int sqlite3_open(const char *filename, sqlite3 **ppDb);
int sqlite3_close(sqlite3 *);
const char *sqlite3_errmsg(sqlite3 *);
int sqlite3_prepare_v2(sqlite3 *db, const char *zSql, int nByte, sqlite3_stmt **ppStmt, const char **pzTail);
int sqlite3_bind_text(sqlite3_stmt *, int, const char *, int, void (*)(void *));
int sqlite3_step(sqlite3_stmt *);
const unsigned char *sqlite3_column_text(sqlite3_stmt *, int iCol);
int sqlite3_finalize(sqlite3_stmt *pStmt);
#ifdef __cplusplus
}
#endif
#endif
