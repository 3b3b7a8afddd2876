import sys

from .simulate import main

sys.exit(main())
