/* Case-correcting forwarder for src/rtDevice/public/IRenderContext.h:3. TEST INFRASTRUCTURE ONLY. */
#include "ShaderCompiler/ShaderFlags.h"
