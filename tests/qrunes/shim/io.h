/* The reference lexer (QRunesParser/lex.yy.cpp) includes the Windows <io.h>;
 * on Linux the functions it needs come from <unistd.h>. */
#include <unistd.h>
