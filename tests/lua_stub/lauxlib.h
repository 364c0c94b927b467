/* Declarations of the Lua 5.4 auxiliary library functions the binding uses
 * (Lua 5.4 reference manual, section 5).  Test infrastructure only. */
#ifndef TM_TEST_LAUXLIB_H
#define TM_TEST_LAUXLIB_H
#include "lua.h"

typedef struct luaL_Reg {
  const char *name;
  lua_CFunction func;
} luaL_Reg;

void *luaL_checkudata(lua_State *L, int arg, const char *tname);
const char *luaL_checklstring(lua_State *L, int arg, size_t *l);
lua_Integer luaL_checkinteger(lua_State *L, int arg);
void luaL_checktype(lua_State *L, int arg, int t);
int luaL_error(lua_State *L, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int luaL_newmetatable(lua_State *L, const char *tname);
void luaL_setfuncs(lua_State *L, const luaL_Reg *l, int nup);

#define luaL_checkstring(L, n) (luaL_checklstring(L, (n), NULL))
#define luaL_getmetatable(L, n) (lua_getfield(L, LUA_REGISTRYINDEX, (n)))
#endif
