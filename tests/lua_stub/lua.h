/* Declarations of the Lua 5.4 C API functions and macros the binding uses,
 * as documented in the Lua 5.4 reference manual (section 4).  Test
 * infrastructure: lets the compile check of the binding run where no Lua
 * headers are installed.  Nothing here is defined; the check only compiles. */
#ifndef TM_TEST_LUA_H
#define TM_TEST_LUA_H
#include <stddef.h>

#define LUA_VERSION_NUM 504
#define LUAI_MAXSTACK 1000000
#define LUA_REGISTRYINDEX (-LUAI_MAXSTACK - 1000)
#define LUA_TNIL 0
#define LUA_TBOOLEAN 1
#define LUA_TNUMBER 3
#define LUA_TSTRING 4
#define LUA_TTABLE 5

typedef struct lua_State lua_State;
typedef long long lua_Integer;
typedef double lua_Number;
typedef ptrdiff_t lua_KContext;
typedef int (*lua_CFunction)(lua_State *L);
typedef int (*lua_KFunction)(lua_State *L, int status, lua_KContext ctx);

int lua_absindex(lua_State *L, int idx);
int lua_gettop(lua_State *L);
void lua_settop(lua_State *L, int idx);
void lua_pushvalue(lua_State *L, int idx);
int lua_type(lua_State *L, int idx);
int lua_isnumber(lua_State *L, int idx);
int lua_toboolean(lua_State *L, int idx);
lua_Number lua_tonumberx(lua_State *L, int idx, int *isnum);
lua_Integer lua_tointegerx(lua_State *L, int idx, int *isnum);
const char *lua_tolstring(lua_State *L, int idx, size_t *len);
void lua_pushinteger(lua_State *L, lua_Integer n);
const char *lua_pushstring(lua_State *L, const char *s);
const char *lua_pushlstring(lua_State *L, const char *s, size_t len);
void lua_pushcclosure(lua_State *L, lua_CFunction fn, int n);
int lua_getfield(lua_State *L, int idx, const char *k);
void lua_setfield(lua_State *L, int idx, const char *k);
void lua_createtable(lua_State *L, int narr, int nrec);
void *lua_newuserdatauv(lua_State *L, size_t sz, int nuvalue);
int lua_setmetatable(lua_State *L, int idx);
int lua_pcallk(lua_State *L, int nargs, int nresults, int msgh, lua_KContext ctx, lua_KFunction k);

#define lua_pop(L, n) lua_settop(L, -(n)-1)
#define lua_newtable(L) lua_createtable(L, 0, 0)
#define lua_newuserdata(L, s) lua_newuserdatauv(L, s, 1)
#define lua_pushcfunction(L, f) lua_pushcclosure(L, (f), 0)
#define lua_isnil(L, n) (lua_type(L, (n)) == LUA_TNIL)
#define lua_tonumber(L, i) lua_tonumberx(L, (i), NULL)
#define lua_tointeger(L, i) lua_tointegerx(L, (i), NULL)
#define lua_tostring(L, i) lua_tolstring(L, (i), NULL)
#define lua_pcall(L, n, r, f) lua_pcallk(L, (n), (r), (f), 0, NULL)
#endif
