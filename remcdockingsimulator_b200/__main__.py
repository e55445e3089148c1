import sys

from .remc import main

sys.exit(main())
