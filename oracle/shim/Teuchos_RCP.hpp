// Stand-in for Teuchos_RCP.hpp: the oracle build uses no reference-counted pointers.
#pragma once
