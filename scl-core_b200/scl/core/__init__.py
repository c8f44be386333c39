from .config import IndexType, RealType, get_config, get_library, get_precision, set_precision  # noqa: F401
from .error import SCLError, check_error  # noqa: F401
from .sparse import BlockStrategy, CsrMatrix  # noqa: F401
